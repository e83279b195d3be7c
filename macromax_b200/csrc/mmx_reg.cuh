// Register-staged FFT passes along a strided axis (the middle passes of the 3D schedule and the axis-0 pass with
// the Green multiply), complex64, power-of-two lengths 64 .. 512.
//
// Same self-sorting stage formulation as mmx_fft.cuh, but the first radix stage reads its butterfly inputs
// straight from global memory into registers and the last stage writes its outputs straight back, so a forward (or
// inverse) pass exchanges data through shared memory only between stages.  A tile is 16 consecutive pencils of one
// outer index; shared memory is laid out [c][j][pencil] with a 16-word (128-byte) row, and every warp covers two
// whole rows in every access, which is conflict-free for 8-byte words.  Thread t works on pencil t % 16, butterfly
// slot (t / 16) % TPP and component t / (16 TPP); a stage with T butterflies per pencil gives each thread T / TPP of
// them.  Global accesses are 16 consecutive words (128 bytes) per row and warp.
#pragma once
#include "mmx_kernels.cuh"

template <int... Rs> struct RegPlanList {};
template <int N> struct RegPlan;
template <> struct RegPlan<64> { using type = RegPlanList<8, 8>; static constexpr int TPP = 8; };
template <> struct RegPlan<128> { using type = RegPlanList<16, 8>; static constexpr int TPP = 8; };
template <> struct RegPlan<256> { using type = RegPlanList<16, 16>; static constexpr int TPP = 16; };
template <> struct RegPlan<512> { using type = RegPlanList<8, 8, 8>; static constexpr int TPP = 32; };
// 192 (vector fields, strided passes only: the 192^3 anisotropic grids): 8 x 8 x 3, 8 threads per pencil
template <> struct RegPlan<192> { using type = RegPlanList<8, 8, 3>; static constexpr int TPP = 8; };

constexpr int kRegP = 16;

// Radix order of the axis-0 pass with the fused Green stage (3-component fields): that stage holds one (pencil,
// butterfly) item per thread, P x N / R of them, so its radix R (the last forward one) must be the largest; for 192
// the radix-3 stage goes first (P x 192 / 8 = 384 items, the block size).
template <int N> struct GreenPlan { using type = typename RegPlan<N>::type; };
template <> struct GreenPlan<192> { using type = RegPlanList<3, 8, 8>; };

template <int C, int N, int P = kRegP> struct RegThreads {
  static constexpr int value = C * P * RegPlan<N>::TPP;
};

// Shared-memory word of row r (= c N + j) and pencil pl in a tile of P pencils.  A 16-pencil row is one 128-byte
// sweep of the banks, so the two rows a warp touches in one access never conflict.  An 8-pencil row is half of one,
// and the four rows of a warp's access are consecutive (stage inputs), 8 apart (the fused Green stage's outputs) or
// 16 apart (a radix-16 stage's outputs): one row of padding after every 16 puts two of them on each half of the
// banks in all three cases.
template <int P> __device__ __forceinline__ int tidx(int r, int pl) {
  if constexpr (P == 16) return r * P + pl;
  else return (r + (r >> 4)) * P + pl;
}
// rows of shared memory that `rows` tile rows take, padding included
template <int P> __host__ __device__ constexpr int tile_rows(int rows) { return P == 16 ? rows : rows + rows / 16; }

// one stage; SRC/DST: 0 = shared memory, 1 = global memory (tile-relative, row stride jstride words)
template <int DIR, int N, int C, int RAD, int L, bool FROM_G, bool TO_G, int P = kRegP>
__device__ __forceinline__ void rstage(float2* __restrict__ sm, const float2* __restrict__ tw, const float2* gsrc,
                                       float2* gdst, int64_t jstride, int64_t cstride) {
  constexpr int TPP = RegPlan<N>::TPP;
  constexpr int T = N / RAD;
  constexpr int NBT = T / TPP;
  static_assert(NBT >= 1 && T % TPP == 0, "stage does not split evenly over the threads");
  constexpr int TSTRIDE = N / (L * RAD);
  const int tid = threadIdx.x;
  const int pl = tid % P;
  const int rest = tid / P;
  const int ii = rest % TPP;
  const int c = rest / TPP;
  float2 u[NBT][RAD];
#pragma unroll
  for (int m = 0; m < NBT; ++m) {
    const int i = ii + m * TPP;
    const int kk = i % L;
#pragma unroll
    for (int q = 0; q < RAD; ++q) {
      const int j = i + q * T;
      if constexpr (FROM_G) u[m][q] = gsrc[c * cstride + (int64_t)j * jstride + pl];
      else u[m][q] = sm[tidx<P>(c * N + j, pl)];
    }
    if constexpr (L > 1) {
#pragma unroll
      for (int q = 1; q < RAD; ++q) {
        float2 w = tw[q * kk * TSTRIDE];
        if (DIR > 0) w = conjc(w);
        u[m][q] = u[m][q] * w;
      }
    }
    bfly<float, RAD, DIR>(u[m], tw, N);
  }
  if constexpr (!FROM_G && !TO_G) __syncthreads();  // in-place shared stage: all reads before any write
#pragma unroll
  for (int m = 0; m < NBT; ++m) {
    const int i = ii + m * TPP;
    const int kk = i % L;
    const int d0 = (i - kk) * RAD + kk;
#pragma unroll
    for (int q = 0; q < RAD; ++q) {
      const int j = d0 + q * L;
      if constexpr (TO_G) gdst[c * cstride + (int64_t)j * jstride + pl] = u[m][q];
      else sm[tidx<P>(c * N + j, pl)] = u[m][q];
    }
  }
  if constexpr (!TO_G) __syncthreads();
}

// all stages of one transform; FIRST_G: first stage reads global; LAST_G: last stage writes global
template <int DIR, int N, int C, bool FIRST_G, bool LAST_G, int P, int L, int R0, int... Rs>
__device__ __forceinline__ void rstages(float2* sm, const float2* tw, const float2* gsrc, float2* gdst, int64_t js,
                                        int64_t cs) {
  constexpr bool last = sizeof...(Rs) == 0;
  rstage<DIR, N, C, R0, L, FIRST_G, LAST_G && last, P>(sm, tw, gsrc, gdst, js, cs);
  if constexpr (!last) rstages<DIR, N, C, false, LAST_G, P, L * R0, Rs...>(sm, tw, gsrc, gdst, js, cs);
}

template <int DIR, int N, int C, bool FIRST_G, bool LAST_G, int P = kRegP, int... Rs>
__device__ __forceinline__ void rfft(float2* sm, const float2* tw, const float2* gsrc, float2* gdst, int64_t js,
                                     int64_t cs, RegPlanList<Rs...>) {
  rstages<DIR, N, C, FIRST_G, LAST_G, P, 1, Rs...>(sm, tw, gsrc, gdst, js, cs);
}

// Radix-plan list algebra: concatenation, reversal, all-but-last and last.
template <class A, class B> struct PlanConcat;
template <int... A, int... B> struct PlanConcat<RegPlanList<A...>, RegPlanList<B...>> {
  using type = RegPlanList<A..., B...>;
};
template <class L> struct PlanReverse;
template <> struct PlanReverse<RegPlanList<>> { using type = RegPlanList<>; };
template <int R0, int... Rs> struct PlanReverse<RegPlanList<R0, Rs...>> {
  using type = typename PlanConcat<typename PlanReverse<RegPlanList<Rs...>>::type, RegPlanList<R0>>::type;
};
template <class L> struct PlanInit;
template <int R0> struct PlanInit<RegPlanList<R0>> { using type = RegPlanList<>; };
template <int R0, int R1, int... Rs> struct PlanInit<RegPlanList<R0, R1, Rs...>> {
  using type = typename PlanConcat<RegPlanList<R0>, typename PlanInit<RegPlanList<R1, Rs...>>::type>::type;
};
template <class L> struct PlanFirst;
template <int R0, int... Rs> struct PlanFirst<RegPlanList<R0, Rs...>> { static constexpr int value = R0; };
// radices whose butterflies use constant coefficients only (no twiddle table)
__host__ __device__ constexpr bool const_coef_radix(int r) {
  return r == 2 || r == 3 || r == 4 || r == 5 || r == 8 || r == 16;
}
template <class L> struct PlanLast;
template <int R0> struct PlanLast<RegPlanList<R0>> { static constexpr int value = R0; };
template <int R0, int R1, int... Rs> struct PlanLast<RegPlanList<R0, R1, Rs...>> {
  static constexpr int value = PlanLast<RegPlanList<R1, Rs...>>::value;
};

// The stages of `List` in order, the first one at span L (FIRST_G: it reads global memory; LAST_G: the last one
// writes global memory).
template <int DIR, int N, int C, bool FIRST_G, bool LAST_G, int L, class List, int P = kRegP> struct RChain;
template <int DIR, int N, int C, bool FIRST_G, bool LAST_G, int L, int P>
struct RChain<DIR, N, C, FIRST_G, LAST_G, L, RegPlanList<>, P> {
  static __device__ __forceinline__ void run(float2*, const float2*, const float2*, float2*, int64_t, int64_t) {}
};
template <int DIR, int N, int C, bool FIRST_G, bool LAST_G, int L, int R0, int... Rs, int P>
struct RChain<DIR, N, C, FIRST_G, LAST_G, L, RegPlanList<R0, Rs...>, P> {
  static __device__ __forceinline__ void run(float2* sm, const float2* tw, const float2* gsrc, float2* gdst,
                                             int64_t js, int64_t cs) {
    constexpr bool last = sizeof...(Rs) == 0;
    rstage<DIR, N, C, R0, L, FIRST_G, LAST_G && last, P>(sm, tw, gsrc, gdst, js, cs);
    RChain<DIR, N, C, false, LAST_G, L * R0, RegPlanList<Rs...>, P>::run(sm, tw, gsrc, gdst, js, cs);
  }
};

// Last forward stage (radix R, span N / R), the scalar Green multiply and the first inverse stage (radix R, span 1)
// of a 16-pencil tile, in registers.  The last forward stage of butterfly i writes the positions i + q N / R, which
// are exactly the inputs of butterfly i of the first inverse stage when the inverse runs the radix plan in reverse
// order; so the spectrum never goes back to shared memory between the two transforms.
//   g(k) = -i a_i / (|k|^2 - a) / N  (solver.py:566-568, with the 1/N of the inverse transform)
template <int N, int R, int P = kRegP>
__device__ __forceinline__ void green_fused_scalar(float2* sm, const float2* tw, const float* sk0, const float* sk1,
                                                   const float* sk2, float ar, float ai, float ai2s, float ais) {
  constexpr int TPP = RegPlan<N>::TPP, T = N / R, NB = T / TPP;
  static_assert(NB >= 1 && T % TPP == 0, "stage does not split evenly over the threads");
  // The stage reads positions i + q T and writes i R + q of the same pencil, so all of a pencil's reads precede its
  // writes.  At 512 samples it runs in NB rounds over P / NB pencils each, one butterfly per thread and round, which
  // keeps the kernel within its register budget; otherwise each thread holds its NB butterflies at once.
  constexpr int ROUNDS = (N == 512) ? NB : 1;
  constexpr int PR = P / ROUNDS;    // pencils per round
  constexpr int NBR = NB / ROUNDS;  // butterflies per thread and round
  const int tid = threadIdx.x;
  const float ai2 = ai * ai;
#pragma unroll 1
  for (int rd = 0; rd < ROUNDS; ++rd) {
    const int pl = rd * PR + tid % PR;
    const int ii = (tid / PR) % (TPP * ROUNDS);
    const float kt2 = sk1[pl] * sk1[pl] + sk2[pl] * sk2[pl];
    float2 u[NBR][R];
#pragma unroll
    for (int m = 0; m < NBR; ++m) {
      const int i = ii + m * TPP * ROUNDS;
#pragma unroll
      for (int q = 0; q < R; ++q) u[m][q] = sm[tidx<P>(i + q * T, pl)];
#pragma unroll
      for (int q = 1; q < R; ++q) u[m][q] = u[m][q] * tw[q * i];
      bfly<float, R, -1>(u[m], tw, N);
#pragma unroll
      for (int q = 0; q < R; ++q) {
        const float k0 = sk0[i + q * T];
        const float dr = fmaf(k0, k0, kt2) - ar;
        const float inv = __fdividef(1.f, fmaf(dr, dr, ai2));
        u[m][q] = u[m][q] * make_float2(ai2s * inv, ais * dr * inv);
      }
      bfly<float, R, +1>(u[m], tw, N);
    }
    __syncthreads();  // every butterfly of these pencils has read its inputs
#pragma unroll
    for (int m = 0; m < NBR; ++m) {
      const int i = ii + m * TPP * ROUNDS;
#pragma unroll
      for (int q = 0; q < R; ++q) sm[tidx<P>(i * R + q, pl)] = u[m][q];
    }
    __syncthreads();
  }
}

// The same fused stage for a 3-component field: one thread takes all three components of a (pencil, butterfly) item,
// so that the dyadic Green multiply (backend/__init__.py:606-649 longitudinal projection, solver.py:571-577) sees
// the whole vector at each k:  F' = g (F - P_L F) + (i alpha_i / alpha) P_L F / N,  P_L = k k^T / |k|^2, with the
// DC rule of the reference (P_L F = F on the grid's axes at k = 0) and no longitudinal part along absent axes.
// The P x (N / R) items are spread over the first threads of the block; the others only join the barriers.
template <int N, int R, int P = kRegP>
__device__ __forceinline__ void green_fused_vector(float2* sm, const float2* tw, const float* sk0, const float* sk1,
                                                   const float* sk2, bool dc_tile, int ndim, float ar, float ai,
                                                   float ai2s, float ais, float2 hs) {
  constexpr int T = N / R, ITEMS = P * T;
  constexpr int THREADS = RegThreads<3, N, P>::value;
  static_assert(ITEMS <= THREADS, "one item per thread");
  const int tid = threadIdx.x;
  const int pl = tid % P;
  const int i = tid / P;
  const bool active = tid < ITEMS;
  float2 u[3][R];
  if (active) {
    const float k1 = sk1[pl], k2 = sk2[pl];
    const float kt2 = k1 * k1 + k2 * k2;
    const float ai2 = ai * ai;
#pragma unroll
    for (int c = 0; c < 3; ++c) {
#pragma unroll
      for (int q = 0; q < R; ++q) u[c][q] = sm[tidx<P>(c * N + i + q * T, pl)];
#pragma unroll
      for (int q = 1; q < R; ++q) u[c][q] = u[c][q] * tw[q * i];
      bfly<float, R, -1>(u[c], tw, N);
    }
#pragma unroll
    for (int q = 0; q < R; ++q) {
      const int j = i + q * T;
      const float k0 = sk0[j];
      const float kk2 = fmaf(k0, k0, kt2);
      const float dr = kk2 - ar;
      const float inv = __fdividef(1.f, fmaf(dr, dr, ai2));
      const float2 g = make_float2(ai2s * inv, ais * dr * inv);
      const float kv[3] = {k0, k1, k2};
      float2 PL[3];
      if (dc_tile && j == 0 && pl == 0) {
#pragma unroll
        for (int c = 0; c < 3; ++c) PL[c] = c < ndim ? u[c][q] : make_float2(0.f, 0.f);
      } else {
        float2 proj = make_float2(0.f, 0.f);
#pragma unroll
        for (int c = 0; c < 3; ++c)
          if (c < ndim) proj += kv[c] * u[c][q];
        proj = proj * __fdividef(1.f, kk2);
#pragma unroll
        for (int c = 0; c < 3; ++c) PL[c] = c < ndim ? kv[c] * proj : make_float2(0.f, 0.f);
      }
#pragma unroll
      for (int c = 0; c < 3; ++c) u[c][q] = g * (u[c][q] - PL[c]) + hs * PL[c];
    }
#pragma unroll
    for (int c = 0; c < 3; ++c) bfly<float, R, +1>(u[c], tw, N);
  }
  __syncthreads();  // every item has read its inputs
  if (active) {
#pragma unroll
    for (int c = 0; c < 3; ++c) {
#pragma unroll
      for (int q = 0; q < R; ++q) sm[tidx<P>(c * N + i * R + q, pl)] = u[c][q];
    }
  }
  __syncthreads();
}

// OPS: OP_FWD (forward pass), OP_INV (inverse pass) or OP_FWD | OP_G | OP_INV (axis-0 pass with the Green multiply)
// resident CTAs per SM the strided passes are compiled for (the register budget follows from it)
#ifndef MMX_REG_MIN_BLOCKS
#define MMX_REG_MIN_BLOCKS 2
#endif
// One-component passes of up to 128 samples (128-thread CTAs: scalar fields, and the component-split FFT-only passes
// of vector fields) are compiled for seven CTAs per SM (72 registers): 115.8 against 116.3 us per 128^3 vector
// iteration and 49.4 against 50.8 us per 128^3 scalar iteration with the unbounded 80-register build; eight CTAs
// (64 registers, spills) were slower.
// The 8-pencil tiles of the vector axis-0 pass (192 threads) run five CTAs per SM at 64 registers (16 bytes of
// spills): 109.6 against 110.7 us per 128^3 vector iteration with four CTAs at 80 registers.
template <int C, int N, int P = kRegP> struct RegMinBlocks {
  static constexpr int value = (C == 1 && N <= 128) ? 896 / RegThreads<C, N, P>::value
                               : P == 8                ? 960 / RegThreads<C, N, P>::value
                                                       : MMX_REG_MIN_BLOCKS;
};
template <int C, int OPS, int N, int P = kRegP>
__global__ void __launch_bounds__(RegThreads<C, N, P>::value, (RegMinBlocks<C, N, P>::value))
    k_reg_pass(IterArgs<float> a) {
  constexpr int THREADS = RegThreads<C, N, P>::value;
  extern __shared__ __align__(16) unsigned char mmx_smem_raw[];
  float2* sm = reinterpret_cast<float2*>(mmx_smem_raw);
  float2* smtw = sm + tile_rows<P>(C * N) * P;
  // component split (one-component kernel on a vector field): blockIdx.y = RHS * csplit + component
  const bool split = C == 1 && a.csplit > 1;
  const int b = split ? (int)blockIdx.y / a.csplit : (int)blockIdx.y;
  const int64_t field0 = split ? (int64_t)blockIdx.y : (int64_t)b * C;  // first component plane of the tile
  const mmx_rhs_state* st = a.st + b;
  const int tid = threadIdx.x;
  const int64_t inner = a.inner;
  const int64_t p0 = (int64_t)blockIdx.x * P;
  const int64_t o = p0 / inner;
  const int64_t in0 = p0 - o * inner;
  // The constant tables -- twiddles and, for the Green passes, the k values of the tile's samples and pencils -- are
  // loaded into registers before the pass waits for its predecessor, and stored to shared memory without a barrier
  // of their own: the first radix stage needs none of them (span 1, constant-coefficient butterflies), and its
  // closing barrier publishes them to the later stages.  A CTA thus waits for one round of global loads (its tile)
  // after the state instead of three.
  constexpr int TWR = (N + THREADS - 1) / THREADS;
  constexpr bool kGreen = (OPS & OP_G) != 0;
  const float2* twg = (const float2*)a.ax.tw;
  float2 twv[TWR];
  float kv0[kGreen ? TWR : 1];
  float kv1 = 0.f, kv2 = 0.f;
#pragma unroll
  for (int k = 0; k < TWR; ++k)
    if (tid + k * THREADS < N) twv[k] = twg[tid + k * THREADS];
  if constexpr (kGreen) {
#pragma unroll
    for (int k = 0; k < TWR; ++k)
      if (tid + k * THREADS < N) kv0[k] = a.kv[0][tid + k * THREADS];
    if (tid < P) {
      const int64_t p = in0 + tid;
      if (a.ndim == 3) {
        const int i1 = (int)(p / a.dims[2]);
        const int i2 = (int)(p - (int64_t)i1 * a.dims[2]);
        kv1 = a.kv[1][i1];
        kv2 = a.kv[2][i2];
      } else if (a.ndim == 2) {
        kv1 = a.kv[1][p];
      }
    }
  }
  pdl_wait();
  pdl_trigger();
  if (!st->active) return;
  float2* tile = a.T + field0 * a.N + o * (int64_t)N * inner + in0;
#pragma unroll
  for (int k = 0; k < TWR; ++k)
    if (tid + k * THREADS < N) smtw[tid + k * THREADS] = twv[k];
  using Plan = typename RegPlan<N>::type;
  static_assert(const_coef_radix(PlanFirst<Plan>::value) &&
                    const_coef_radix(PlanFirst<typename GreenPlan<N>::type>::value),
                "the first stage must not read the twiddle table (it is published by that stage's barrier)");
  if constexpr (OPS == OP_FWD) {
    rfft<-1, N, C, true, true, P>(sm, smtw, tile, tile, inner, a.N, Plan{});
  } else if constexpr (OPS == OP_INV) {
    rfft<+1, N, C, true, true, P>(sm, smtw, tile, tile, inner, a.N, Plan{});
  } else {
    __shared__ float sk1[P], sk2[P], sk0[N];
    const ChiCoef<float> cc = chi_coef<float>(st);
    if constexpr (C == 1) {
      // scalar field: k tables first, then the forward stages but the last, the fused last-forward / Green /
      // first-inverse stage, and the remaining inverse stages in reverse radix order
      if (tid < P) {
        sk1[tid] = kv1;
        sk2[tid] = kv2;
      }
#pragma unroll
      for (int k = 0; k < TWR; ++k)
        if (tid + k * THREADS < N) sk0[tid + k * THREADS] = kv0[k];
      // (the forward chain's first stage reads global memory only; its closing barrier publishes the tables)
      using Init = typename PlanInit<Plan>::type;
      constexpr int RL = PlanLast<Plan>::value;
      RChain<-1, N, 1, true, false, 1, Init, P>::run(sm, smtw, tile, tile, inner, a.N);
      const float ar = cc.alpha_re, ai = cc.alpha_im;
      green_fused_scalar<N, RL, P>(sm, smtw, sk0, sk1, sk2, ar, ai, ai * ai * a.inv_total, -ai * a.inv_total);
      RChain<+1, N, 1, false, true, RL, typename PlanReverse<Init>::type, P>::run(sm, smtw, tile, tile, inner, a.N);
      return;
    } else if constexpr (C == 3 && (N == 128 || N == 192)) {
      // vector field: the same fused schedule with the dyadic Green multiply (all three components per item)
      if (tid < P) {
        sk1[tid] = kv1;
        sk2[tid] = kv2;
      }
#pragma unroll
      for (int k = 0; k < TWR; ++k)
        if (tid + k * THREADS < N) sk0[tid + k * THREADS] = kv0[k];
      using GPlan = typename GreenPlan<N>::type;
      using Init = typename PlanInit<GPlan>::type;
      constexpr int RL = PlanLast<GPlan>::value;
      RChain<-1, N, 3, true, false, 1, Init, P>::run(sm, smtw, tile, tile, inner, a.N);
      const float ar = cc.alpha_re, ai = cc.alpha_im;
      const float2 hs = divc(make_float2(0.f, ai), make_float2(ar, ai)) * a.inv_total;
      green_fused_vector<N, RL, P>(sm, smtw, sk0, sk1, sk2, in0 == 0, a.ndim, ar, ai, ai * ai * a.inv_total,
                                   -ai * a.inv_total, hs);
      RChain<+1, N, 3, false, true, RL, typename PlanReverse<Init>::type, P>::run(sm, smtw, tile, tile, inner,
                                                                                   a.N);
      return;
    }
    // forward transform into shared memory, Green multiply, inverse transform back to global memory
    rfft<-1, N, C, true, false, P>(sm, smtw, tile, tile, inner, a.N, Plan{});
    if (tid < P) {
      sk1[tid] = kv1;
      sk2[tid] = kv2;
    }
#pragma unroll
    for (int k = 0; k < TWR; ++k)
      if (tid + k * THREADS < N) sk0[tid + k * THREADS] = kv0[k];
    __syncthreads();
    const float ar = cc.alpha_re, ai = cc.alpha_im;
    const float2 hs = divc(make_float2(0.f, ai), make_float2(ar, ai)) * a.inv_total;
    const float ai2s = ai * ai * a.inv_total, ais = -ai * a.inv_total;
    for (int e = tid; e < N * P; e += THREADS) {
      const int pl = e % P;
      const int j = e / P;
      const float k0 = sk0[j], k1 = sk1[pl], k2 = sk2[pl];
      const float kk2 = k0 * k0 + k1 * k1 + k2 * k2;
      const float dr = kk2 - ar;
      const float inv = __fdividef(1.f, fmaf(dr, dr, ai * ai));
      const float2 g = make_float2(ai2s * inv, ais * dr * inv);  // -i a_i / (|k|^2 - a) / N
      if constexpr (C == 1) {
        sm[tidx<P>(j, pl)] = sm[tidx<P>(j, pl)] * g;
      } else {
        float2 F[3], PL[3];
        const float kv[3] = {k0, k1, k2};
#pragma unroll
        for (int c = 0; c < 3; ++c) F[c] = sm[tidx<P>(c * N + j, pl)];
        if (j == 0 && in0 + pl == 0) {
#pragma unroll
          for (int c = 0; c < 3; ++c) PL[c] = c < a.ndim ? F[c] : make_float2(0.f, 0.f);
        } else {
          float2 proj = make_float2(0.f, 0.f);
#pragma unroll
          for (int c = 0; c < 3; ++c)
            if (c < a.ndim) proj += kv[c] * F[c];
          proj = proj * __fdividef(1.f, kk2);
#pragma unroll
          for (int c = 0; c < 3; ++c) PL[c] = c < a.ndim ? kv[c] * proj : make_float2(0.f, 0.f);
        }
#pragma unroll
        for (int c = 0; c < 3; ++c) sm[tidx<P>(c * N + j, pl)] = g * (F[c] - PL[c]) + hs * PL[c];
      }
    }
    __syncthreads();
    rfft<+1, N, C, false, true, P>(sm, smtw, tile, tile, inner, a.N, Plan{});
  }
}

// ---------------------------------------------------------------------------------------------------------------
// Register-staged passes along the contiguous axis with the fused prologue / epilogue (isotropic chi).
//
// A tile is PC consecutive rows (pencils of N contiguous samples).  Thread t works on butterfly slot t % TPP,
// row (t / TPP) % PC and component t / (TPP PC), so consecutive threads touch consecutive samples of a row in the
// first-stage loads and the last-stage stores.  Shared memory is [c][row][N + N/16] with sample m stored at
// m + m/16: with that skew the stride-RAD scatter of a stage and the unit-stride gather of the next one both hit
// every bank pair exactly twice per warp (the minimum for 8-byte words).
//   PRO | FWD: x = chi(alpha) E + s'(alpha) computed as the first stage loads it; forward FFT; T written back.
//   INV | EPI: inverse FFT of T; the last stage produces the transformed samples in registers and applies
//              d = chi(alpha)(T - E), E' = E + d, with FP64 partial norms, directly against global memory.
// ---------------------------------------------------------------------------------------------------------------
template <int C, int N> struct RegCDefault {
  static constexpr int TPP = RegPlan<N>::TPP;
  // prologue and epilogue tiles: at most 256 threads per CTA, several CTAs per SM
  static constexpr int P0 = 256 / (C * TPP);
  static constexpr int PC = P0 >= 32 ? 32 : P0 >= 16 ? 16 : P0 >= 8 ? 8 : P0 >= 4 ? 4 : P0 >= 2 ? 2 : 1;
  static constexpr int PC_EPI = PC;  // (four-row tiles for the 128-sample vector epilogue measured slower)
  // persistent variant (one CTA per SM, stages its inputs in shared memory): 384-thread budget, half the rows
  static constexpr int PP0 = 384 / (C * TPP);
  static constexpr int PC_PIPE0 = PP0 >= 32 ? 32 : PP0 >= 16 ? 16 : PP0 >= 8 ? 8 : PP0 >= 4 ? 4 : PP0 >= 2 ? 2 : 1;
  static constexpr int PC_PIPE = PC_PIPE0 >= 2 ? PC_PIPE0 / 2 : 1;
};

template <int C, int N, int PC_> struct RegC {
  static constexpr int TPP = RegPlan<N>::TPP;
  static constexpr int PC = PC_;
  static constexpr int THREADS = C * PC * TPP;
  static constexpr int PITCH = N + N / 16;
  static __device__ __forceinline__ int idx(int c, int row, int m) { return (c * PC + row) * PITCH + m + (m >> 4); }
};

// bounded wait on an mbarrier phase; returns false if the copy did not complete within `limit` polls
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, unsigned parity, int limit = 1 << 20) {
  const unsigned addr = (unsigned)__cvta_generic_to_shared(bar);
  for (int it = 0; it < limit; ++it) {
    unsigned done;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(done)
        : "r"(addr), "r"(parity)
        : "memory");
    if (done) return true;
  }
  return false;
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, unsigned count) {
  const unsigned addr = (unsigned)__cvta_generic_to_shared(bar);
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(addr), "r"(count) : "memory");
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, unsigned bytes) {
  const unsigned addr = (unsigned)__cvta_generic_to_shared(bar);
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(addr), "r"(bytes) : "memory");
}

// one bulk global -> shared copy (16-byte aligned addresses, size a multiple of 16), completing on the mbarrier
__device__ __forceinline__ void bulk_load(void* smem_dst, const void* gsrc, unsigned bytes, uint64_t* bar) {
  const unsigned d = (unsigned)__cvta_generic_to_shared(smem_dst);
  const unsigned b = (unsigned)__cvta_generic_to_shared(bar);
  asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(d),
               "l"(gsrc), "r"(bytes), "r"(b)
               : "memory");
}


// in-place shared-memory stage for the contiguous layout
template <int DIR, int N, int C, int PC_, int RAD, int L>
__device__ __forceinline__ void cstage_smem(float2* __restrict__ sm, const float2* __restrict__ tw) {
  using G = RegC<C, N, PC_>;
  constexpr int TPP = G::TPP, PC = G::PC;
  constexpr int T = N / RAD;
  constexpr int NBT = T / TPP;
  constexpr int TSTRIDE = N / (L * RAD);
  const int tid = threadIdx.x;
  const int ii = tid % TPP;
  const int row = (tid / TPP) % PC;
  const int c = tid / (TPP * PC);
  float2 u[NBT][RAD];
#pragma unroll
  for (int m = 0; m < NBT; ++m) {
    const int i = ii + m * TPP;
    const int kk = i % L;
#pragma unroll
    for (int q = 0; q < RAD; ++q) u[m][q] = sm[G::idx(c, row, i + q * T)];
    if constexpr (L > 1) {
#pragma unroll
      for (int q = 1; q < RAD; ++q) {
        float2 w = tw[q * kk * TSTRIDE];
        if (DIR > 0) w = conjc(w);
        u[m][q] = u[m][q] * w;
      }
    }
    bfly<float, RAD, DIR>(u[m], tw, N);
  }
  __syncthreads();
#pragma unroll
  for (int m = 0; m < NBT; ++m) {
    const int i = ii + m * TPP;
    const int kk = i % L;
    const int d0 = (i - kk) * RAD + kk;
#pragma unroll
    for (int q = 0; q < RAD; ++q) sm[G::idx(c, row, d0 + q * L)] = u[m][q];
  }
  __syncthreads();
}

template <int... Rs> struct RadixInfo;
template <int R0, int... Rs> struct RadixInfo<R0, Rs...> {
  static constexpr int first = R0;
  static constexpr int count = 1 + sizeof...(Rs);
};
template <int... Rs> struct LastRadix;
template <int R0> struct LastRadix<R0> { static constexpr int value = R0; };
template <int R0, int R1, int... Rs> struct LastRadix<R0, R1, Rs...> {
  static constexpr int value = LastRadix<R1, Rs...>::value;
};

// middle stages of a plan (all but first and last), starting at L = first radix
template <int DIR, int N, int C, int PC, int L, int... Rs> struct CMidOfPlan;
template <int DIR, int N, int C, int PC, int L, int R0> struct CMidOfPlan<DIR, N, C, PC, L, R0> {
  static __device__ __forceinline__ void run(float2*, const float2*) {}
};
template <int DIR, int N, int C, int PC, int L, int R0, int R1, int... Rs>
struct CMidOfPlan<DIR, N, C, PC, L, R0, R1, Rs...> {
  static __device__ __forceinline__ void run(float2* sm, const float2* tw) {
    cstage_smem<DIR, N, C, PC, R0, L>(sm, tw);
    CMidOfPlan<DIR, N, C, PC, L * R0, R1, Rs...>::run(sm, tw);
  }
};

template <class PL> struct RegPlanArgs;
template <int... Rs> struct RegPlanArgs<RegPlanList<Rs...>> {
  static constexpr int R_first = RadixInfo<Rs...>::first;
  static constexpr int R_last = LastRadix<Rs...>::value;
  static constexpr int count = RadixInfo<Rs...>::count;
  template <int DIR, int N, int C, int PC> static __device__ __forceinline__ void mid(float2* sm, const float2* tw) {
    // stages 2 .. count-1 (skip the first, stop before the last)
    MidHelper<DIR, N, C, PC, Rs...>::run(sm, tw);
  }
  template <int DIR, int N, int C, int PC, int R0, int... Rest> struct MidHelper {
    static __device__ __forceinline__ void run(float2* sm, const float2* tw) {
      CMidOfPlan<DIR, N, C, PC, R0, Rest...>::run(sm, tw);
    }
  };
};

// Resident CTAs per SM the register budget is sized for: MMX_REGC_THREADS_PER_SM threads per SM (1024 by default,
// i.e. 64 registers per thread).
#ifndef MMX_REGC_THREADS_PER_SM
#define MMX_REGC_THREADS_PER_SM 1024
#endif
template <int C, int OPS, int N, int PC_> struct RegCMinBlocks {
  static constexpr int T = RegC<C, N, PC_>::THREADS;
  static constexpr int value = MMX_REGC_THREADS_PER_SM / T >= 2 ? MMX_REGC_THREADS_PER_SM / T : 2;
};

template <int C, int OPS, int N, int PC_>
__global__ void __launch_bounds__(RegC<C, N, PC_>::THREADS, (RegCMinBlocks<C, OPS, N, PC_>::value))
    k_regc_pass(IterArgs<float> a) {
  using G = RegC<C, N, PC_>;
  using PA = RegPlanArgs<typename RegPlan<N>::type>;
  constexpr int TPP = G::TPP, PC = G::PC, THREADS = G::THREADS;
  extern __shared__ __align__(16) unsigned char mmx_smem_raw[];
  float2* sm = reinterpret_cast<float2*>(mmx_smem_raw);
  float2* smtw = sm + C * PC * G::PITCH;
  const int b = blockIdx.y;
  const mmx_rhs_state* st = a.st + b;
  if (threadIdx.x == 0) {
    // inputs no kernel writes (chi, and s' for the prologue): prefetch them into L2 before waiting for the
    // previous pass; the fields follow once the state says which buffer is current
    const int64_t row0 = (int64_t)blockIdx.x * PC * N;
    const unsigned chunk = (unsigned)(PC * N * sizeof(float2));
    prefetch_l2(a.chi + row0, chunk);
    if constexpr ((OPS & OP_PRO) != 0) {
#pragma unroll
      for (int cc2 = 0; cc2 < C; ++cc2)
        if (!source_is_zero(st, cc2)) prefetch_l2(a.src + ((int64_t)b * C + cc2) * a.N + row0, chunk);
    }
  }
  // the twiddle table is constant: loaded into registers before the wait, stored to shared memory after it with no
  // barrier of its own (both first stages use constant-coefficient butterflies; their closing barriers publish it)
  constexpr int TWR = (N + THREADS - 1) / THREADS;
  static_assert(const_coef_radix(PA::R_first), "the first stage must not read the twiddle table");
  const float2* twg = (const float2*)a.ax.tw;
  float2 twv[TWR];
#pragma unroll
  for (int k = 0; k < TWR; ++k)
    if ((int)threadIdx.x + k * THREADS < N) twv[k] = twg[threadIdx.x + k * THREADS];
  pdl_wait();
  pdl_trigger();
  if (!st->active) return;
  const ChiCoef<float> cc = chi_coef<float>(st);
  const int tid = threadIdx.x;
  const int ii = tid % TPP;
  const int row = (tid / TPP) % PC;
  const int c = tid / (TPP * PC);
  const int64_t N3 = a.N;
  const int64_t fbase = (int64_t)b * C * N3;
  const int64_t rowbase = ((int64_t)blockIdx.x * PC + row) * N;  // voxel index of sample 0 of this row
  const int cur = st->cur;
  const float2* __restrict__ Ecur = cur ? a.E1 : a.E0;
  float2* __restrict__ Eoth = cur ? a.E0 : a.E1;
#pragma unroll
  for (int k = 0; k < TWR; ++k)
    if (tid + k * THREADS < N) smtw[tid + k * THREADS] = twv[k];

  if constexpr (OPS == (OP_PRO | OP_FWD)) {
    // E, s' and chi of the tile's rows are contiguous chunks: prefetch them into L2 in bulk
    if (tid == 0) {
      const int64_t row0 = (int64_t)blockIdx.x * PC * N;
      const unsigned chunk = (unsigned)(PC * N * sizeof(float2));
#pragma unroll
      for (int cc2 = 0; cc2 < C; ++cc2) prefetch_l2(Ecur + fbase + cc2 * N3 + row0, chunk);
    }
    // first stage: x = chi E + s' from global, radix R_first, L = 1, outputs to shared memory, one butterfly at a
    // time (the source is global memory, so each butterfly can be stored as soon as it is done)
    constexpr int RAD = PA::R_first;
    constexpr int T = N / RAD;
    constexpr int NBT = T / TPP;
    const float2* __restrict__ eS = Ecur + fbase + c * N3 + rowbase;
    const float2* __restrict__ sS = a.src + fbase + c * N3 + rowbase;
    const float2* __restrict__ xS = a.chi + rowbase;
    const bool with_src = !source_is_zero(st, c);  // uniform over the component's warps
#pragma unroll 1
    for (int m = 0; m < NBT; ++m) {
      const int i = ii + m * TPP;
      float2 u[RAD];
#pragma unroll
      for (int q = 0; q < RAD; ++q) {
        const int s_ = i + q * T;
        u[q] = (cc.a * xS[s_] + cc.b) * eS[s_];
        if (with_src) u[q] += cc.s * sS[s_];
      }
      bfly<float, RAD, -1>(u, smtw, N);
#pragma unroll
      for (int q = 0; q < RAD; ++q) sm[G::idx(c, row, i * RAD + q)] = u[q];
    }
    __syncthreads();
    PA::template mid<-1, N, C, PC>(sm, smtw);
    // last stage: shared -> registers -> T (global), one butterfly at a time
    constexpr int RL = PA::R_last;
    constexpr int TL = N / RL;
    constexpr int NBL = TL / TPP;
    constexpr int LL = N / RL;
    float2* __restrict__ tO = a.T + fbase + c * N3 + rowbase;
#pragma unroll 1
    for (int m = 0; m < NBL; ++m) {
      const int i = ii + m * TPP;
      float2 v[RL];
#pragma unroll
      for (int q = 0; q < RL; ++q) v[q] = sm[G::idx(c, row, i + q * TL)];
#pragma unroll
      for (int q = 1; q < RL; ++q) v[q] = v[q] * smtw[q * i];
      bfly<float, RL, -1>(v, smtw, N);
#pragma unroll
      for (int q = 0; q < RL; ++q) tO[i + q * LL] = v[q];
    }
  } else {
    // INV | EPI.  E and chi of the tile's rows are contiguous chunks (PC rows x N samples per component): a bulk
    // L2 prefetch issued now brings them on chip while the inverse transform of T runs; the last stage then reads
    // them with plain loads.
    if (tid == 0) {
      const int64_t row0 = (int64_t)blockIdx.x * PC * N;
      const unsigned chunk = (unsigned)(PC * N * sizeof(float2));
#pragma unroll
      for (int cc2 = 0; cc2 < C; ++cc2) prefetch_l2(Ecur + fbase + cc2 * N3 + row0, chunk);
    }
    // first stage from T (global) into shared memory
    constexpr int RAD = PA::R_first;
    constexpr int T = N / RAD;
    constexpr int NBT = T / TPP;
    float2 u[NBT][RAD];
#pragma unroll
    for (int m = 0; m < NBT; ++m) {
      const int i = ii + m * TPP;
#pragma unroll
      for (int q = 0; q < RAD; ++q) u[m][q] = a.T[fbase + c * N3 + rowbase + i + q * T];
      bfly<float, RAD, +1>(u[m], smtw, N);
    }
#pragma unroll
    for (int m = 0; m < NBT; ++m) {
      const int i = ii + m * TPP;
#pragma unroll
      for (int q = 0; q < RAD; ++q) sm[G::idx(c, row, i * RAD + q)] = u[m][q];
    }
    __syncthreads();
    PA::template mid<+1, N, C, PC>(sm, smtw);
    constexpr int RL = PA::R_last;
    constexpr int TL = N / RL;
    constexpr int NBL = TL / TPP;
    constexpr int LL = N / RL;
    double dd2 = 0.0, en2 = 0.0;
    const float2* __restrict__ eS = Ecur + fbase + c * N3 + rowbase;
    const float2* __restrict__ xS = a.chi + rowbase;
    float2* __restrict__ eO = Eoth + fbase + c * N3 + rowbase;
    // one butterfly at a time: its RL outputs, then RL epilogue words, keep the live registers low
#pragma unroll 1
    for (int m = 0; m < NBL; ++m) {
      const int i = ii + m * TPP;
      float2 v[RL];
#pragma unroll
      for (int q = 0; q < RL; ++q) v[q] = sm[G::idx(c, row, i + q * TL)];
#pragma unroll
      for (int q = 1; q < RL; ++q) v[q] = v[q] * conjc(smtw[q * i]);
      bfly<float, RL, +1>(v, smtw, N);
#pragma unroll
      for (int q = 0; q < RL; ++q) {
        const int s_ = i + q * LL;
        const float2 e = eS[s_];
        const float2 x = cc.a * xS[s_] + cc.b;
        const float2 d = x * (v[q] - e);
        const float2 en = e + d;
        eO[s_] = en;
        dd2 += norm2d(d);
        en2 += norm2d(en);
      }
    }
    finish_pass_norms(a, b, dd2, en2);
  }
}

// ---------------------------------------------------------------------------------------------------------------
// Contiguous prologue / epilogue passes for a 3x3 chi (MMX_CHI_SYM6 or MMX_CHI_MAT3) on a 3-component field, for
// rows whose first radix stage has exactly C TPP butterflies (192 = 8 x 8 x 3: 24 per row).  The matrix couples
// the components at each voxel, so the stages that apply it give one thread all three components of a butterfly
// slot: the prologue's first stage forms (chi E + s')_c for c = 0..2 at the slot's samples (each E, s' and chi word
// loaded once) and runs three butterflies; the epilogue reads the inverse transform of all three components back
// from shared memory and forms d = chi (T - E) per sample.  The middle and the other outer stage keep the
// per-component layout of k_regc_pass.
// ---------------------------------------------------------------------------------------------------------------
template <int CHI> __device__ __forceinline__ int chi_entry(int r, int s) {
  if constexpr (CHI == MMX_CHI_SYM6) {
    constexpr int K6[9] = {0, 1, 2, 1, 3, 4, 2, 4, 5};
    return K6[r * 3 + s];
  } else {
    return r * 3 + s;
  }
}

// The prologue of one tile (PC rows) of right-hand side b for a 3x3 chi: x = chi(alpha) E + s'(alpha) formed as the
// first radix stage loads it (one thread per (row, butterfly slot), all three components), the forward FFT along
// the contiguous axis, written to T.  Expects the twiddles in smtw and the tile's shared memory free.
template <int N, int PC_, int CHI>
__device__ __forceinline__ void aniso_pro_tile(const IterArgs<float>& a, int b, int64_t tile, float2* sm,
                                               const float2* smtw, const ChiCoef<float>& cc, const float2* Ecur) {
  constexpr int C = 3;
  using G = RegC<C, N, PC_>;
  using PA = RegPlanArgs<typename RegPlan<N>::type>;
  constexpr int TPP = G::TPP, PC = G::PC;
  constexpr int M = CHI == MMX_CHI_SYM6 ? 6 : 9;
  constexpr int RAD = PA::R_first;
  constexpr int T1 = N / RAD;
  static_assert(T1 == C * TPP, "one (row, butterfly slot) item per thread");
  constexpr int RL = PA::R_last;
  constexpr int TL = N / RL;
  constexpr int NBL = TL / TPP;
  const mmx_rhs_state* st = a.st + b;
  const int tid = threadIdx.x;
  const int ii = tid % TPP;
  const int row = (tid / TPP) % PC;
  const int c = tid / (TPP * PC);
  const int irow = tid / T1;
  const int islot = tid % T1;
  const int64_t N3 = a.N;
  const int64_t fbase = (int64_t)b * C * N3;
  const int64_t ibase = (tile * PC + irow) * N;
  const float2* __restrict__ eI = Ecur + fbase + ibase;
  const float2* __restrict__ xI = a.chi + ibase;
  const float2* __restrict__ sI = a.src + fbase + ibase;
  float2 u[C][RAD];
#pragma unroll
  for (int q = 0; q < RAD; ++q) {
    const int s_ = islot + q * T1;
    float2 e[C], m[M];
#pragma unroll
    for (int r = 0; r < C; ++r) e[r] = eI[r * N3 + s_];
#pragma unroll
    for (int k = 0; k < M; ++k) m[k] = cc.a * xI[k * N3 + s_];
#pragma unroll
    for (int r = 0; r < C; ++r) {
      float2 acc = cc.b * e[r];
      if (!source_is_zero(st, r)) acc += cc.s * sI[r * N3 + s_];
#pragma unroll
      for (int s2 = 0; s2 < C; ++s2) acc += m[chi_entry<CHI>(r, s2)] * e[s2];
      u[r][q] = acc;
    }
  }
#pragma unroll
  for (int r = 0; r < C; ++r) {
    bfly<float, RAD, -1>(u[r], smtw, N);
#pragma unroll
    for (int q = 0; q < RAD; ++q) sm[G::idx(r, irow, islot * RAD + q)] = u[r][q];
  }
  __syncthreads();
  PA::template mid<-1, N, C, PC>(sm, smtw);
  float2* __restrict__ tO = a.T + fbase + c * N3 + (tile * PC + row) * N;
#pragma unroll 1
  for (int mm = 0; mm < NBL; ++mm) {
    const int i = ii + mm * TPP;
    float2 v[RL];
#pragma unroll
    for (int q = 0; q < RL; ++q) v[q] = sm[G::idx(c, row, i + q * TL)];
#pragma unroll
    for (int q = 1; q < RL; ++q) v[q] = v[q] * smtw[q * i];
    bfly<float, RL, -1>(v, smtw, N);
#pragma unroll
    for (int q = 0; q < RL; ++q) tO[i + q * TL] = v[q];
  }
}

template <int OPS, int N, int PC_, int CHI>
__global__ void __launch_bounds__(RegC<3, N, PC_>::THREADS, 4) k_regc_aniso_pass(IterArgs<float> a) {
  constexpr int C = 3;
  using G = RegC<C, N, PC_>;
  using PA = RegPlanArgs<typename RegPlan<N>::type>;
  constexpr int TPP = G::TPP, PC = G::PC, THREADS = G::THREADS;
  constexpr int M = CHI == MMX_CHI_SYM6 ? 6 : 9;
  constexpr int RAD = PA::R_first;
  constexpr int T1 = N / RAD;  // first-stage butterflies per row
  static_assert(T1 == C * TPP, "one (row, butterfly slot) item per thread");
  extern __shared__ __align__(16) unsigned char mmx_smem_raw[];
  float2* sm = reinterpret_cast<float2*>(mmx_smem_raw);
  float2* smtw = sm + C * PC * G::PITCH;
  const int b = blockIdx.y;
  const mmx_rhs_state* st = a.st + b;
  const int64_t N3 = a.N;
  // (no L2 bulk prefetch here: with 12 words per voxel of 8 rows in flight per CTA it evicted data still to be
  // read; 644 instead of 664 us per 192^3 iteration without it)
  pdl_wait();
  pdl_trigger();
  if (!st->active) return;
  const ChiCoef<float> cc = chi_coef<float>(st);
  const int tid = threadIdx.x;
  const int ii = tid % TPP;          // per-component layout (FFT stages)
  const int row = (tid / TPP) % PC;
  const int c = tid / (TPP * PC);
  const int irow = tid / T1;         // all-component layout (chi stages): row and butterfly slot
  const int islot = tid % T1;
  const int64_t fbase = (int64_t)b * C * N3;
  const int cur = st->cur;
  const float2* __restrict__ Ecur = cur ? a.E1 : a.E0;
  float2* __restrict__ Eoth = cur ? a.E0 : a.E1;
  const float2* twg = (const float2*)a.ax.tw;
  for (int t = tid; t < N; t += THREADS) smtw[t] = twg[t];
  __syncthreads();
  const int64_t ibase = ((int64_t)blockIdx.x * PC + irow) * N;  // voxel of sample 0 of the item's row
  const float2* __restrict__ eI = Ecur + fbase + ibase;          // component r at eI[r N3 + sample]
  const float2* __restrict__ xI = a.chi + ibase;                 // entry k at xI[k N3 + sample]
  constexpr int RL = PA::R_last;
  constexpr int TL = N / RL;
  constexpr int NBL = TL / TPP;

  if constexpr (OPS == (OP_PRO | OP_FWD)) {
    aniso_pro_tile<N, PC_, CHI>(a, b, blockIdx.x, sm, smtw, cc, Ecur);
  } else {
    // INV | EPI: the inverse transform in the per-component layout, its outputs back in shared memory at their
    // natural positions, then the epilogue in the all-component layout
    constexpr int NBT = T1 / TPP;
    const float2* __restrict__ tI = a.T + fbase + c * N3 + ((int64_t)blockIdx.x * PC + row) * N;
#pragma unroll 1
    for (int mm = 0; mm < NBT; ++mm) {
      const int i = ii + mm * TPP;
      float2 v[RAD];
#pragma unroll
      for (int q = 0; q < RAD; ++q) v[q] = tI[i + q * T1];
      bfly<float, RAD, +1>(v, smtw, N);
#pragma unroll
      for (int q = 0; q < RAD; ++q) sm[G::idx(c, row, i * RAD + q)] = v[q];
    }
    __syncthreads();
    PA::template mid<+1, N, C, PC>(sm, smtw);
#pragma unroll 1
    for (int mm = 0; mm < NBL; ++mm) {
      const int i = ii + mm * TPP;
      float2 v[RL];
#pragma unroll
      for (int q = 0; q < RL; ++q) v[q] = sm[G::idx(c, row, i + q * TL)];
#pragma unroll
      for (int q = 1; q < RL; ++q) v[q] = v[q] * conjc(smtw[q * i]);
      bfly<float, RL, +1>(v, smtw, N);
#pragma unroll
      for (int q = 0; q < RL; ++q) sm[G::idx(c, row, i + q * TL)] = v[q];  // the positions this thread read
    }
    __syncthreads();
    double dd2 = 0.0, en2 = 0.0;
    float2* __restrict__ eO = Eoth + fbase + ibase;
#pragma unroll 2
    for (int q = 0; q < N / T1; ++q) {
      const int s_ = islot + q * T1;
      float2 e[C], diff[C], m[M];
#pragma unroll
      for (int r = 0; r < C; ++r) {
        e[r] = eI[r * N3 + s_];
        diff[r] = sm[G::idx(r, irow, s_)] - e[r];
      }
#pragma unroll
      for (int k = 0; k < M; ++k) m[k] = cc.a * xI[k * N3 + s_];
#pragma unroll
      for (int r = 0; r < C; ++r) {
        float2 d = cc.b * diff[r];
#pragma unroll
        for (int s2 = 0; s2 < C; ++s2) d += m[chi_entry<CHI>(r, s2)] * diff[s2];
        const float2 en = e[r] + d;
        eO[r * N3 + s_] = en;
        dd2 += norm2d(d);
        en2 += norm2d(en);
      }
    }
    finish_pass_norms(a, b, dd2, en2);
  }
}

// ---------------------------------------------------------------------------------------------------------------
// Persistent, double-buffered variants of the contiguous prologue / epilogue passes.
//
// Each CTA walks the tiles blockIdx.x, blockIdx.x + gridDim.x, ... of all right-hand sides.  The inputs of a tile
// (PRO: E, chi, s'; EPI: T, E, chi -- PC rows of N contiguous samples per component) arrive by bulk copies, one per
// row, into shared rows of pitch N + 8 words (the 64-byte skew keeps the 4-rows-per-warp reads conflict-free),
// completing on the stage's mbarrier.  While a tile is transformed, the copies of the CTA's next-but-one tile are
// already in flight in the other stage, so DRAM traffic does not stop during the arithmetic.  Waits are bounded:
// on a timeout the tile is computed from global memory instead and MMX_STATUS_TIMEOUT is raised.
// ---------------------------------------------------------------------------------------------------------------
template <int C, int OPS, int N, int PC> struct PipeLayout {
  static constexpr int RP = N + 8;                                  // staged row pitch (words)
  static constexpr int NIN = (OPS & OP_PRO) ? (2 * C + 1) : (2 * C + 1);  // PRO: E, s', chi; EPI: T, E, chi
  static constexpr int STAGE = NIN * PC * RP;                       // words per stage
  static constexpr int WORK = C * PC * RegC<C, N, PC>::PITCH;
  static constexpr size_t bytes() { return (size_t)(WORK + N + 2 * STAGE) * sizeof(float2); }
};

template <int C, int OPS, int N, int PC>
__global__ void __launch_bounds__(RegC<C, N, PC>::THREADS, 1) k_pipe_pass(IterArgs<float> a, int tiles_per_rhs) {
  using G = RegC<C, N, PC>;
  using L = PipeLayout<C, OPS, N, PC>;
  using PA = RegPlanArgs<typename RegPlan<N>::type>;
  constexpr int TPP = G::TPP, THREADS = G::THREADS, RP = L::RP;
  extern __shared__ __align__(16) unsigned char mmx_smem_raw[];
  float2* sm = reinterpret_cast<float2*>(mmx_smem_raw);
  float2* smtw = sm + L::WORK;
  float2* stage0 = smtw + N;
  __shared__ __align__(8) uint64_t bars[2];
  __shared__ int s_active[2], s_cur[2];
  const int tid = threadIdx.x;
  const int ii = tid % TPP;
  const int row = (tid / TPP) % PC;
  const int c = tid / (TPP * PC);
  const int64_t N3 = a.N;
  const int nrhs = a.nrhs;
  const int64_t ntiles = (int64_t)tiles_per_rhs * nrhs;
  const float2* twg = (const float2*)a.ax.tw;
  for (int t = tid; t < N; t += THREADS) smtw[t] = twg[t];
  const unsigned rowbytes = (unsigned)(N * sizeof(float2));

  // input k of a tile (PRO: 0..C-1 = E_c, C..2C-1 = s'_c, 2C = chi; EPI: 0..C-1 = T_c, C..2C-1 = E_c, 2C = chi)
  auto issue = [&](int s, int64_t t) {
    const int b = (int)(t / tiles_per_rhs);
    const int64_t row0 = (t % tiles_per_rhs) * PC;
    const mmx_rhs_state* st = a.st + b;
    const int active = st->active;
    s_active[s] = active;
    s_cur[s] = st->cur;
    if (!active) {  // keep the stage's mbarrier phases in step with the tile sequence: complete this phase now
      mbar_expect_tx(&bars[s], 0u);
      return;
    }
    const float2* Ecur = st->cur ? a.E1 : a.E0;
    const int64_t fbase = (int64_t)b * C * N3;
    float2* dst = stage0 + s * L::STAGE;
    mbar_expect_tx(&bars[s], rowbytes * (unsigned)(L::NIN * PC));
    for (int k = 0; k < L::NIN; ++k) {
      const float2* src;
      if ((OPS & OP_PRO) != 0) src = k < C ? Ecur + fbase + k * N3 : (k < 2 * C ? a.src + fbase + (k - C) * N3 : a.chi);
      else src = k < C ? a.T + fbase + k * N3 : (k < 2 * C ? Ecur + fbase + (k - C) * N3 : a.chi);
      for (int r = 0; r < PC; ++r) bulk_load(dst + (k * PC + r) * RP, src + (row0 + r) * N, rowbytes, &bars[s]);
    }
  };

  if (tid == 0) {
    mbar_init(&bars[0], 1);
    mbar_init(&bars[1], 1);
    if ((int64_t)blockIdx.x < ntiles) issue(0, blockIdx.x);
    if ((int64_t)blockIdx.x + gridDim.x < ntiles) issue(1, blockIdx.x + gridDim.x);
  }
  __syncthreads();

  int kk = 0;
  for (int64_t t = blockIdx.x; t < ntiles; t += gridDim.x, ++kk) {
    const int s = kk & 1;
    const unsigned parity = (unsigned)((kk >> 1) & 1);
    const int b = (int)(t / tiles_per_rhs);
    const int64_t rowbase = ((t % tiles_per_rhs) * PC + row) * N;
    const mmx_rhs_state* st = a.st + b;
    const int64_t fbase = (int64_t)b * C * N3;
    if (s_active[s]) {
      const ChiCoef<float> cc = chi_coef<float>(st);
      const int cur = s_cur[s];
      const float2* Ecur = cur ? a.E1 : a.E0;
      float2* Eoth = cur ? a.E0 : a.E1;
      const bool staged = mbar_wait(&bars[s], parity, a.poll_limit);
      if (!staged && tid == 0) atomicOr(&const_cast<mmx_rhs_state*>(st)->status, MMX_STATUS_TIMEOUT);
      const float2* stg = stage0 + s * L::STAGE;
      if constexpr ((OPS & OP_PRO) != 0) {
        constexpr int RAD = PA::R_first;
        constexpr int T = N / RAD;
        constexpr int NBT = T / TPP;
        float2 u[NBT][RAD];
#pragma unroll
        for (int m = 0; m < NBT; ++m) {
          const int i = ii + m * TPP;
#pragma unroll
          for (int q = 0; q < RAD; ++q) {
            const int smp = i + q * T;
            float2 e, sv, xv;
            if (staged) {
              e = stg[(c * PC + row) * RP + smp];
              sv = stg[((C + c) * PC + row) * RP + smp];
              xv = stg[(2 * C * PC + row) * RP + smp];
            } else {
              e = Ecur[fbase + c * N3 + rowbase + smp];
              sv = a.src[fbase + c * N3 + rowbase + smp];
              xv = a.chi[rowbase + smp];
            }
            u[m][q] = (cc.a * xv + cc.b) * e + cc.s * sv;
          }
          bfly<float, RAD, -1>(u[m], smtw, N);
        }
#pragma unroll
        for (int m = 0; m < NBT; ++m) {
          const int i = ii + m * TPP;
#pragma unroll
          for (int q = 0; q < RAD; ++q) sm[G::idx(c, row, i * RAD + q)] = u[m][q];
        }
        __syncthreads();
        PA::template mid<-1, N, C, PC>(sm, smtw);
        constexpr int RL = PA::R_last;
        constexpr int TL = N / RL;
        constexpr int NBL = TL / TPP;
        constexpr int LL = N / RL;
        float2 v[NBL][RL];
#pragma unroll
        for (int m = 0; m < NBL; ++m) {
          const int i = ii + m * TPP;
#pragma unroll
          for (int q = 0; q < RL; ++q) v[m][q] = sm[G::idx(c, row, i + q * TL)];
#pragma unroll
          for (int q = 1; q < RL; ++q) v[m][q] = v[m][q] * smtw[q * i];
          bfly<float, RL, -1>(v[m], smtw, N);
#pragma unroll
          for (int q = 0; q < RL; ++q) a.T[fbase + c * N3 + rowbase + i + q * LL] = v[m][q];
        }
        __syncthreads();  // stage buffer and work area free for reuse
      } else {
        constexpr int RAD = PA::R_first;
        constexpr int T = N / RAD;
        constexpr int NBT = T / TPP;
        float2 u[NBT][RAD];
#pragma unroll
        for (int m = 0; m < NBT; ++m) {
          const int i = ii + m * TPP;
#pragma unroll
          for (int q = 0; q < RAD; ++q) {
            const int smp = i + q * T;
            u[m][q] = staged ? stg[(c * PC + row) * RP + smp] : a.T[fbase + c * N3 + rowbase + smp];
          }
          bfly<float, RAD, +1>(u[m], smtw, N);
        }
#pragma unroll
        for (int m = 0; m < NBT; ++m) {
          const int i = ii + m * TPP;
#pragma unroll
          for (int q = 0; q < RAD; ++q) sm[G::idx(c, row, i * RAD + q)] = u[m][q];
        }
        __syncthreads();
        PA::template mid<+1, N, C, PC>(sm, smtw);
        constexpr int RL = PA::R_last;
        constexpr int TL = N / RL;
        constexpr int NBL = TL / TPP;
        constexpr int LL = N / RL;
        double dd2 = 0.0, en2 = 0.0;
        float2 v[NBL][RL];
#pragma unroll
        for (int m = 0; m < NBL; ++m) {
          const int i = ii + m * TPP;
#pragma unroll
          for (int q = 0; q < RL; ++q) v[m][q] = sm[G::idx(c, row, i + q * TL)];
#pragma unroll
          for (int q = 1; q < RL; ++q) v[m][q] = v[m][q] * conjc(smtw[q * i]);
          bfly<float, RL, +1>(v[m], smtw, N);
#pragma unroll
          for (int q = 0; q < RL; ++q) {
            const int smp = i + q * LL;
            float2 e, xv;
            if (staged) {
              e = stg[((C + c) * PC + row) * RP + smp];
              xv = stg[(2 * C * PC + row) * RP + smp];
            } else {
              e = Ecur[fbase + c * N3 + rowbase + smp];
              xv = a.chi[rowbase + smp];
            }
            const float2 d = (cc.a * xv + cc.b) * (v[m][q] - e);
            const float2 en = e + d;
            Eoth[fbase + c * N3 + rowbase + smp] = en;
            dd2 += norm2d(d);
            en2 += norm2d(en);
          }
        }
        // per-tile partial norms and the fused decision (the block-wide reduction synchronises the block)
        {
          __shared__ int s_last;
          double out2[2];
          block_reduce_2<float>(dd2, en2, out2);
          if (tid == 0) {
            double* dst = a.partials + ((int64_t)b * tiles_per_rhs + (t % tiles_per_rhs)) * 2;
            dst[0] = out2[0];
            dst[1] = out2[1];
            __threadfence();
            const unsigned prev = atomicAdd(a.done + b, 1u);
            s_last = (prev == (unsigned)tiles_per_rhs - 1);
          }
          __syncthreads();
          if (s_last) {
            __threadfence();
            decide_rhs(const_cast<mmx_rhs_state*>(st), a.partials + (int64_t)b * tiles_per_rhs * 2, tiles_per_rhs);
            if (tid == 0) a.done[b] = 0u;
          }
          __syncthreads();
        }
      }
      if (!staged && tid == 0) mbar_wait(&bars[s], parity);  // drain before the stage is re-armed
    } else if (tid == 0) {
      mbar_wait(&bars[s], parity);  // the phase was completed without copies
    }
    // refill this stage with the tile two steps ahead
    if (tid == 0) {
      const int64_t nxt = t + 2 * (int64_t)gridDim.x;
      if (nxt < ntiles) issue(s, nxt);
    }
    __syncthreads();
  }
}
