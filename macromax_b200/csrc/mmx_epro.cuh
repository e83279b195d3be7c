// Epilogue of iteration k fused with the prologue of iteration k + 1 (contiguous axis, complex64, isotropic chi).
//
// Per iteration the unfused schedule streams the field twice through the contiguous-axis passes: the epilogue reads
// E and writes E' = E + chi (T - E), and the next iteration's prologue reads E' back to form chi E' + s'.  Here the
// epilogue pass goes on with the values it holds in registers:
//
//   k_regc_epro:   inverse FFT of T along the contiguous axis, E' = E + chi (T - E) with the partial norms, then
//                  x = chi E' + s' and the forward FFT of x, written to T  -- the next iteration's first pass.
//
// The forward transform runs the radix plan in reverse order, so its first stage (radix R_last, span 1) reads
// exactly the positions i + q N / R_last at which the inverse transform's last stage left its outputs: that stage
// is done in registers, straight after the epilogue, and only the later stages go through shared memory.
//
// The prologue is speculative.  chi(alpha) E' + s'(alpha) is the next iteration's input only if the divergence
// guard accepts E' (the usual case); it is taken at the end of the same pass by the last CTA of each right-hand
// side.  If it rejects, the next input is chi(alpha') E + s'(alpha') with the old field and alpha' = alpha with its
// imaginary part raised (solver.py:1090-1094), and k_regc_repair recomputes the prologue pass for that right-hand
// side.  The repair pass is a grid-stride loop that leaves at once for every right-hand side whose update was
// accepted (or that is no longer active), so on the common path it costs one short launch.
#pragma once
#include "mmx_reg.cuh"

// Stages of `List` on the contiguous layout, the first one at span L; all but the last run in shared memory, the
// last one (span N / R) writes this thread's row of the destination in global memory.
template <int DIR, int N, int C, int PC, int L, class List> struct CChainToGlobal;
template <int DIR, int N, int C, int PC, int L, int R0>
struct CChainToGlobal<DIR, N, C, PC, L, RegPlanList<R0>> {
  static __device__ __forceinline__ void run(float2* sm, const float2* tw, float2* __restrict__ grow) {
    using G = RegC<C, N, PC>;
    constexpr int TPP = G::TPP, T = N / R0, NB = T / TPP;
    static_assert(L * R0 == N, "the last stage spans the whole line");
    static_assert(NB >= 1 && T % TPP == 0, "stage does not split evenly over the threads");
    const int tid = threadIdx.x;
    const int ii = tid % TPP;
    const int row = (tid / TPP) % PC;
    const int c = tid / (TPP * PC);
#pragma unroll 1
    for (int m = 0; m < NB; ++m) {
      const int i = ii + m * TPP;  // i < T = L, so the twiddle exponent is q i
      float2 v[R0];
#pragma unroll
      for (int q = 0; q < R0; ++q) v[q] = sm[G::idx(c, row, i + q * T)];
#pragma unroll
      for (int q = 1; q < R0; ++q) {
        float2 w = tw[q * i];
        if (DIR > 0) w = conjc(w);
        v[q] = v[q] * w;
      }
      bfly<float, R0, DIR>(v, tw, N);
#pragma unroll
      for (int q = 0; q < R0; ++q) grow[i + q * T] = v[q];
    }
  }
};
template <int DIR, int N, int C, int PC, int L, int R0, int R1, int... Rs>
struct CChainToGlobal<DIR, N, C, PC, L, RegPlanList<R0, R1, Rs...>> {
  static __device__ __forceinline__ void run(float2* sm, const float2* tw, float2* __restrict__ grow) {
    cstage_smem<DIR, N, C, PC, R0, L>(sm, tw);
    CChainToGlobal<DIR, N, C, PC, L * R0, RegPlanList<R1, Rs...>>::run(sm, tw, grow);
  }
};

// The prologue pass for the tile `tile` of right-hand side b: x = chi(alpha) E + s'(alpha) on the load, forward FFT
// along the contiguous axis, written to T (the same work as k_regc_pass<C, PRO | FWD>).
template <int C, int N, int PC>
__device__ __forceinline__ void regc_pro_tile(const IterArgs<float>& a, int b, int64_t tile, float2* sm,
                                              const float2* smtw, const ChiCoef<float>& cc, const float2* Ecur) {
  using G = RegC<C, N, PC>;
  using PA = RegPlanArgs<typename RegPlan<N>::type>;
  constexpr int TPP = G::TPP;
  const int tid = threadIdx.x;
  const int ii = tid % TPP;
  const int row = (tid / TPP) % PC;
  const int c = tid / (TPP * PC);
  const int64_t N3 = a.N;
  const int64_t fbase = (int64_t)b * C * N3;
  const int64_t rowbase = (tile * PC + row) * N;
  constexpr int RAD = PA::R_first;
  constexpr int T = N / RAD;
  constexpr int NBT = T / TPP;
  const float2* __restrict__ eS = Ecur + fbase + c * N3 + rowbase;
  const float2* __restrict__ sS = a.src + fbase + c * N3 + rowbase;
  const float2* __restrict__ xS = a.chi + rowbase;
  const bool with_src = !source_is_zero(a.st + b, c);
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
}

// The fused pass holds the first forward stage of all its butterflies across a barrier: it is sized for 960 threads
// per SM (five 192-thread CTAs of the 128-sample vector pass, up to 68 registers per thread).  Measured on the 128^3
// vector iteration: 122.9 us with five CTAs per SM against 125.2 us with four (768 threads, 80 registers).
#ifndef MMX_EPRO_THREADS_PER_SM
#define MMX_EPRO_THREADS_PER_SM 960
#endif
template <int C, int N, int PC> struct EproMinBlocks {
  static constexpr int T = RegC<C, N, PC>::THREADS;
  static constexpr int value = MMX_EPRO_THREADS_PER_SM / T >= 2 ? MMX_EPRO_THREADS_PER_SM / T : 2;
};

template <int C, int N, int PC>
__global__ void __launch_bounds__(RegC<C, N, PC>::THREADS, (EproMinBlocks<C, N, PC>::value))
    k_regc_epro(IterArgs<float> a) {
  using G = RegC<C, N, PC>;
  using Plan = typename RegPlan<N>::type;
  using PA = RegPlanArgs<Plan>;
  constexpr int TPP = G::TPP, THREADS = G::THREADS;
  extern __shared__ __align__(16) unsigned char mmx_smem_raw[];
  float2* sm = reinterpret_cast<float2*>(mmx_smem_raw);
  float2* smtw = sm + C * PC * G::PITCH;
  const int b = blockIdx.y;
  const mmx_rhs_state* st = a.st + b;
  const int64_t N3 = a.N;
  const int64_t row0 = (int64_t)blockIdx.x * PC * N;
  const unsigned chunk = (unsigned)(PC * N * sizeof(float2));
  if (threadIdx.x == 0) {  // inputs no kernel writes: chi and s'
    prefetch_l2(a.chi + row0, chunk);
#pragma unroll
    for (int cc2 = 0; cc2 < C; ++cc2)
      if (!source_is_zero(st, cc2)) prefetch_l2(a.src + ((int64_t)b * C + cc2) * N3 + row0, chunk);
  }
  // the twiddle table is constant: loaded into registers before the wait, stored to shared memory after it with no
  // barrier of its own (the first inverse stage uses constant-coefficient butterflies only; its closing barrier
  // publishes the table)
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
  const int64_t fbase = (int64_t)b * C * N3;
  const int64_t rowbase = ((int64_t)blockIdx.x * PC + row) * N;
  const int cur = st->cur;
  const float2* __restrict__ Ecur = cur ? a.E1 : a.E0;
  float2* __restrict__ Eoth = cur ? a.E0 : a.E1;
  if (tid == 0) {
#pragma unroll
    for (int cc2 = 0; cc2 < C; ++cc2) prefetch_l2(Ecur + fbase + cc2 * N3 + row0, chunk);
  }
#pragma unroll
  for (int k = 0; k < TWR; ++k)
    if (tid + k * THREADS < N) smtw[tid + k * THREADS] = twv[k];

  // inverse transform of T: first stage from global memory, middle stages in shared memory
  float2* __restrict__ trow = a.T + fbase + c * N3 + rowbase;
  {
    constexpr int RAD = PA::R_first;
    constexpr int T = N / RAD;
    constexpr int NBT = T / TPP;
#pragma unroll 1
    for (int m = 0; m < NBT; ++m) {
      const int i = ii + m * TPP;
      float2 u[RAD];
#pragma unroll
      for (int q = 0; q < RAD; ++q) u[q] = trow[i + q * T];
      bfly<float, RAD, +1>(u, smtw, N);
#pragma unroll
      for (int q = 0; q < RAD; ++q) sm[G::idx(c, row, i * RAD + q)] = u[q];
    }
  }
  __syncthreads();
  PA::template mid<+1, N, C, PC>(sm, smtw);

  // last inverse stage, epilogue, speculative prologue and the first forward stage, in registers
  constexpr int RL = PA::R_last;
  constexpr int TL = N / RL;
  constexpr int NBL = TL / TPP;
  constexpr int LL = N / RL;
  const float2* __restrict__ eS = Ecur + fbase + c * N3 + rowbase;
  const float2* __restrict__ sS = a.src + fbase + c * N3 + rowbase;
  const float2* __restrict__ xS = a.chi + rowbase;
  float2* __restrict__ eO = Eoth + fbase + c * N3 + rowbase;
  const bool with_src = !source_is_zero(st, c);  // uniform over the component's warps
  double dd2 = 0.0, en2 = 0.0;
  // Two-stage plans (64, 128, 256 samples): the first forward stage writes its outputs y[i][k1] (k1 < RL) to the
  // positions i + LL k1 that its inputs came from, so no barrier separates the last inverse stage's reads from these
  // writes, and nothing is held in registers across one.  The last forward stage then reads, for its butterfly k1,
  // y[i][k1] at i + LL k1 (i < N / RL): the butterflies and twiddles of the self-sorting stage pair, with the
  // intermediate stored at other positions (114.8 against 115.7 us per 128^3 vector iteration; the iterates agree
  // to complex64 rounding, 5e-7 after 20 iterations).  Longer plans keep the self-sorting layout.
  constexpr bool kInPlace = PA::count == 2;
  float2 xf[kInPlace ? 1 : NBL][RL];
#pragma unroll
  for (int m = 0; m < NBL; ++m) {
    const int i = ii + m * TPP;
    float2 v[RL];
#pragma unroll
    for (int q = 0; q < RL; ++q) v[q] = sm[G::idx(c, row, i + q * TL)];
#pragma unroll
    for (int q = 1; q < RL; ++q) v[q] = v[q] * conjc(smtw[q * i]);
    bfly<float, RL, +1>(v, smtw, N);
    float2* x_m = xf[kInPlace ? 0 : m];
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
      x_m[q] = x * en;  // next iteration's chi(alpha) E' + s'(alpha), if E' is accepted
      if (with_src) x_m[q] += cc.s * sS[s_];
    }
    bfly<float, RL, -1>(x_m, smtw, N);  // first forward stage of the reversed plan (span 1)
    if constexpr (kInPlace) {
#pragma unroll
      for (int q = 0; q < RL; ++q) sm[G::idx(c, row, i + q * LL)] = x_m[q];  // positions this thread read
    }
  }
  if constexpr (kInPlace) {
    __syncthreads();
    constexpr int R0 = N / RL;     // radix of the last forward stage (the plan's first radix)
    constexpr int NB0 = RL / TPP;  // its butterflies per thread
    static_assert(NB0 >= 1 && RL % TPP == 0, "last forward stage does not split evenly over the threads");
#pragma unroll 1
    for (int mm = 0; mm < NB0; ++mm) {
      const int k1 = ii + mm * TPP;
      float2 u[R0];
#pragma unroll
      for (int q = 0; q < R0; ++q) u[q] = sm[G::idx(c, row, q + LL * k1)];
#pragma unroll
      for (int q = 1; q < R0; ++q) u[q] = u[q] * smtw[q * k1];
      bfly<float, R0, -1>(u, smtw, N);
#pragma unroll
      for (int q = 0; q < R0; ++q) trow[k1 + RL * q] = u[q];
    }
  } else {
    __syncthreads();  // every thread has read its inputs of the last inverse stage
#pragma unroll
    for (int m = 0; m < NBL; ++m) {
      const int i = ii + m * TPP;
#pragma unroll
      for (int q = 0; q < RL; ++q) sm[G::idx(c, row, i * RL + q)] = xf[m][q];
    }
    __syncthreads();
    CChainToGlobal<-1, N, C, PC, RL, typename PlanReverse<typename PlanInit<Plan>::type>::type>::run(sm, smtw,
                                                                                                   trow);
  }
  finish_pass_norms(a, b, dd2, en2);
}

// Prologue pass again for every right-hand side whose last update the divergence guard rejected (the fused pass
// above computed it from the rejected field).  Grid-stride over the tiles of each such right-hand side.
template <int C, int N, int PC>
__global__ void __launch_bounds__(RegC<C, N, PC>::THREADS, (RegCMinBlocks<C, OP_PRO | OP_FWD, N, PC>::value))
    k_regc_repair(IterArgs<float> a, int tiles_per_rhs) {
  using G = RegC<C, N, PC>;
  constexpr int THREADS = G::THREADS;
  extern __shared__ __align__(16) unsigned char mmx_smem_raw[];
  float2* sm = reinterpret_cast<float2*>(mmx_smem_raw);
  float2* smtw = sm + C * PC * G::PITCH;
  const float2* twg = (const float2*)a.ax.tw;
  for (int t = threadIdx.x; t < N; t += THREADS) smtw[t] = twg[t];
  pdl_wait();
  pdl_trigger();
  __syncthreads();
  for (int b = 0; b < a.nrhs; ++b) {
    const mmx_rhs_state* st = a.st + b;
    if (!st->active || st->accepted) continue;  // uniform over the CTA
    const ChiCoef<float> cc = chi_coef<float>(st);
    const float2* Ecur = st->cur ? a.E1 : a.E0;
    for (int64_t t = blockIdx.x; t < tiles_per_rhs; t += gridDim.x) {
      regc_pro_tile<C, N, PC>(a, b, t, sm, smtw, cc, Ecur);
      __syncthreads();  // the tile's shared memory is free again
    }
  }
}

// ---------------------------------------------------------------------------------------------------------------
// The same fusion for a 3x3 chi (MMX_CHI_SYM6 / MMX_CHI_MAT3) on rows of k_regc_aniso_pass's lengths (192).
//
// The epilogue stage of k_regc_aniso_pass already gives one thread all three components of a voxel and the voxel's
// chi entries, so after E' = E + chi (T - E) the thread forms the next iteration's input x = chi(alpha) E' + s'
// from the same chi words (the operations in the order of the prologue's) and writes it over the inverse
// transform's output, at the positions it has just read.  The forward transform then runs from shared memory in
// the per-component layout and its last stage writes T.  Per voxel and iteration the six (or nine) chi words and E'
// are read once instead of twice, and one pass over the grid is saved.  The prologue is speculative as above;
// k_regc_aniso_repair redoes it for a right-hand side whose update was rejected.
// ---------------------------------------------------------------------------------------------------------------
// Measured on the 192^3 anisotropic iteration (582.8 us against 617.8 us for the plain passes): four 192-thread CTAs
// per SM at 80 registers.  Five CTAs (64 registers: spills) took 664-700 us; three CTAs with the chi stage unrolled
// four times 613 us; the first inverse stage's loads all issued at once 592 us; L2 bulk prefetches of the tile's chi,
// s' and E rows 587-590 us.
template <int N, int PC_, int CHI>
__global__ void __launch_bounds__(RegC<3, N, PC_>::THREADS, 4) k_regc_aniso_epro(IterArgs<float> a) {
  constexpr int C = 3;
  using G = RegC<C, N, PC_>;
  using Plan = typename RegPlan<N>::type;
  using PA = RegPlanArgs<Plan>;
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
  // the twiddle table is constant: loaded into registers before the wait, stored to shared memory after it with no
  // barrier of its own (the first inverse stage's butterflies use constant coefficients; its closing barrier
  // publishes the table)
  constexpr int TWR = (N + THREADS - 1) / THREADS;
  static_assert(const_coef_radix(RAD), "the first stage must not read the twiddle table");
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
  const int ii = tid % TPP;          // per-component layout (FFT stages)
  const int row = (tid / TPP) % PC;
  const int c = tid / (TPP * PC);
  const int irow = tid / T1;         // all-component layout (chi stage): row and butterfly slot
  const int islot = tid % T1;
  const int64_t fbase = (int64_t)b * C * N3;
  const int cur = st->cur;
  const float2* __restrict__ Ecur = cur ? a.E1 : a.E0;
  float2* __restrict__ Eoth = cur ? a.E0 : a.E1;
#pragma unroll
  for (int k = 0; k < TWR; ++k)
    if (tid + k * THREADS < N) smtw[tid + k * THREADS] = twv[k];
  const int64_t ibase = ((int64_t)blockIdx.x * PC + irow) * N;  // voxel of sample 0 of the item's row
  const float2* __restrict__ eI = Ecur + fbase + ibase;          // component r at eI[r N3 + sample]
  const float2* __restrict__ xI = a.chi + ibase;                 // entry k at xI[k N3 + sample]
  const float2* __restrict__ sI = a.src + fbase + ibase;
  float2* __restrict__ eO = Eoth + fbase + ibase;
  float2* __restrict__ trow = a.T + fbase + c * N3 + ((int64_t)blockIdx.x * PC + row) * N;
  constexpr int RL = PA::R_last;
  constexpr int TL = N / RL;
  constexpr int NBL = TL / TPP;
  // inverse transform of T: first stage from global memory, middle stages, last stage back to the positions it read
  {
    constexpr int NBT = T1 / TPP;
#pragma unroll 1
    for (int mm = 0; mm < NBT; ++mm) {
      const int i = ii + mm * TPP;
      float2 v[RAD];
#pragma unroll
      for (int q = 0; q < RAD; ++q) v[q] = trow[i + q * T1];
      bfly<float, RAD, +1>(v, smtw, N);
#pragma unroll
      for (int q = 0; q < RAD; ++q) sm[G::idx(c, row, i * RAD + q)] = v[q];
    }
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
    for (int q = 0; q < RL; ++q) sm[G::idx(c, row, i + q * TL)] = v[q];
  }
  __syncthreads();
  // epilogue and speculative prologue, all three components of a voxel per thread
  bool with_src[C];
#pragma unroll
  for (int r = 0; r < C; ++r) with_src[r] = !source_is_zero(st, r);
  double dd2 = 0.0, en2 = 0.0;
#pragma unroll 2
  for (int q = 0; q < N / T1; ++q) {
    const int s_ = islot + q * T1;
    float2 e[C], diff[C], en[C], m[M];
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
      en[r] = e[r] + d;
      eO[r * N3 + s_] = en[r];
      dd2 += norm2d(d);
      en2 += norm2d(en[r]);
    }
#pragma unroll
    for (int r = 0; r < C; ++r) {
      float2 acc = cc.b * en[r];
      if (with_src[r]) acc += cc.s * sI[r * N3 + s_];
#pragma unroll
      for (int s2 = 0; s2 < C; ++s2) acc += m[chi_entry<CHI>(r, s2)] * en[s2];
      sm[G::idx(r, irow, s_)] = acc;  // a position this thread has read above
    }
  }
  __syncthreads();
  CChainToGlobal<-1, N, C, PC, 1, Plan>::run(sm, smtw, trow);
  finish_pass_norms(a, b, dd2, en2);
}

// Prologue pass again, for a 3x3 chi, for every right-hand side whose last update was rejected (grid-stride over
// its tiles; the CTAs leave at once when every update was accepted).
template <int N, int PC_, int CHI>
__global__ void __launch_bounds__(RegC<3, N, PC_>::THREADS, 4) k_regc_aniso_repair(IterArgs<float> a,
                                                                                   int tiles_per_rhs) {
  using G = RegC<3, N, PC_>;
  constexpr int THREADS = G::THREADS;
  extern __shared__ __align__(16) unsigned char mmx_smem_raw[];
  float2* sm = reinterpret_cast<float2*>(mmx_smem_raw);
  float2* smtw = sm + 3 * G::PC * G::PITCH;
  const float2* twg = (const float2*)a.ax.tw;
  for (int t = threadIdx.x; t < N; t += THREADS) smtw[t] = twg[t];
  pdl_wait();
  pdl_trigger();
  __syncthreads();
  for (int b = 0; b < a.nrhs; ++b) {
    const mmx_rhs_state* st = a.st + b;
    if (!st->active || st->accepted) continue;  // uniform over the CTA
    const ChiCoef<float> cc = chi_coef<float>(st);
    const float2* Ecur = st->cur ? a.E1 : a.E0;
    for (int64_t t = blockIdx.x; t < tiles_per_rhs; t += gridDim.x) {
      aniso_pro_tile<N, PC_, CHI>(a, b, t, sm, smtw, cc, Ecur);
      __syncthreads();  // the tile's shared memory is free again
    }
  }
}
