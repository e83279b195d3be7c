// Compile-time specialised FFT pass kernels for the common axis lengths (64 .. 1024).
//
// Same algorithm and data flow as k_iter_pass (mmx_kernels.cuh) but with the transform length, radix plan, tile
// width and thread count fixed at compile time, so that every index computation folds into shifts, masks and
// multiplications by constants, the stages are straight-line code, the twiddle table sits in shared memory and
// global traffic uses 16-byte accesses (two consecutive complex64 words per access).  A pass tile is P pencils
// x N samples x C components.  Strided axes (inner > 1) need P | inner, so a tile is P consecutive pencils of one
// outer index; the contiguous axis (inner == 1) takes P consecutive rows.
#pragma once
#include "mmx_kernels.cuh"

template <int... Rs> struct RadixList {};

template <int N> struct FastPlan;
template <> struct FastPlan<64> { using type = RadixList<8, 8>; };
template <> struct FastPlan<128> { using type = RadixList<16, 8>; };
template <> struct FastPlan<192> { using type = RadixList<3, 8, 8>; };
template <> struct FastPlan<256> { using type = RadixList<16, 16>; };
template <> struct FastPlan<384> { using type = RadixList<3, 16, 8>; };
template <> struct FastPlan<512> { using type = RadixList<8, 8, 8>; };
template <> struct FastPlan<1024> { using type = RadixList<16, 8, 8>; };

template <class R, int DIR, int N, int C, int P, int SP, int THREADS, int RAD, int L>
__device__ __forceinline__ void cstage(cpx<R>* __restrict__ sm, const cpx<R>* __restrict__ tw) {
  constexpr int T = N / RAD;
  constexpr int NB = C * P * T;
  constexpr int MAXB = (NB + THREADS - 1) / THREADS;
  constexpr int TSTRIDE = N / (L * RAD);
  const int tid = threadIdx.x;
  cpx<R> u[MAXB][RAD];
  int dst[MAXB];
#pragma unroll
  for (int k = 0; k < MAXB; ++k) {
    const int b = tid + k * THREADS;
    dst[k] = -1;
    if ((NB % THREADS == 0) || b < NB) {
      const int pl = b % P;
      const int rest = b / P;
      const int i = rest % T;
      const int c = rest / T;
      const int kk = i % L;
      const int base = (c * N) * SP + pl;
#pragma unroll
      for (int q = 0; q < RAD; ++q) u[k][q] = sm[base + (i + q * T) * SP];
      if (L > 1) {
#pragma unroll
        for (int q = 1; q < RAD; ++q) {
          cpx<R> w = tw[q * kk * TSTRIDE];
          if (DIR > 0) w = conjc(w);
          u[k][q] = u[k][q] * w;
        }
      }
      bfly<R, RAD, DIR>(u[k], tw, N);
      dst[k] = base + ((i - kk) * RAD + kk) * SP;
    }
  }
  __syncthreads();
#pragma unroll
  for (int k = 0; k < MAXB; ++k) {
    if ((NB % THREADS == 0) || dst[k] >= 0) {
#pragma unroll
      for (int q = 0; q < RAD; ++q) sm[dst[k] + q * L * SP] = u[k][q];
    }
  }
  __syncthreads();
}

template <class R, int DIR, int N, int C, int P, int SP, int THREADS, int L>
__device__ __forceinline__ void cstages(cpx<R>*, const cpx<R>*, RadixList<>) {}

template <class R, int DIR, int N, int C, int P, int SP, int THREADS, int L, int R0, int... Rs>
__device__ __forceinline__ void cstages(cpx<R>* sm, const cpx<R>* tw, RadixList<R0, Rs...>) {
  cstage<R, DIR, N, C, P, SP, THREADS, R0, L>(sm, tw);
  cstages<R, DIR, N, C, P, SP, THREADS, L * R0>(sm, tw, RadixList<Rs...>{});
}

template <class R, int DIR, int N, int C, int P, int SP, int THREADS>
__device__ __forceinline__ void cfft_tile(cpx<R>* sm, const cpx<R>* tw) {
  cstages<R, DIR, N, C, P, SP, THREADS, 1>(sm, tw, typename FastPlan<N>::type{});
}

// threads of a specialised pass: EPT = 8 complex words per thread per stage on average
template <int C, int N, int P> struct FastThreads {
  static constexpr int value = (C * N * P) / 8 < 64 ? 64 : ((C * N * P) / 8 > 512 ? 512 : (C * N * P) / 8);
};

template <int C, int CHI, int OPS, int N, int P, bool STRIDED>
__global__ void __launch_bounds__(FastThreads<C, N, P>::value, 2) k_fast_pass(IterArgs<float> a) {
  using R = float;
  constexpr int THREADS = FastThreads<C, N, P>::value;
  constexpr int SP = P > 1 ? P + 1 : 1;
  constexpr int ELEMS = C * N * P;
  extern __shared__ __align__(16) unsigned char mmx_smem_raw[];
  float2* sm = reinterpret_cast<float2*>(mmx_smem_raw);
  float2* smtw = sm + C * N * SP;  // twiddle table copy [N]
  const int b = blockIdx.y;
  const mmx_rhs_state* st = a.st + b;
  pdl_wait();
  pdl_trigger();
  if (!st->active) return;
  const ChiCoef<R> cc = chi_coef<R>(st);
  const int tid = threadIdx.x;
  const int64_t N3 = a.N;
  const int64_t inner = a.inner;
  const int64_t fbase = (int64_t)b * C * N3;
  const int cur = st->cur;
  float2* __restrict__ Ecur = cur ? a.E1 : a.E0;
  float2* __restrict__ Eoth = cur ? a.E0 : a.E1;
  // tile origin: strided: P consecutive pencils of one outer index; contiguous: P consecutive rows
  int64_t tile_base;  // address of (pencil 0, sample 0) of the tile, component 0
  int64_t in0 = 0;    // first inner index (strided)
  {
    const int64_t p0 = (int64_t)blockIdx.x * P;
    if (STRIDED) {
      const int64_t o = p0 / inner;
      in0 = p0 - o * inner;
      tile_base = o * (int64_t)N * inner + in0;
    } else {
      tile_base = p0 * N;
    }
  }
  const int64_t jstride = STRIDED ? inner : 1;  // address step along the transform axis
  constexpr int pstride_c = STRIDED ? 1 : N;    // address step between pencils (contiguous case)
  const cpx<R>* __restrict__ twg = (const cpx<R>*)a.ax.tw;
  for (int t = tid; t < N; t += THREADS) smtw[t] = twg[t];
  if constexpr (!STRIDED && (OPS & (OP_PRO | OP_EPI)) != 0) {
    // the tile's P rows are contiguous chunks of chi, E (and s'): bring them into L2 in bulk while the first loads
    // are in flight (the epilogue's T is still in L2 from the previous pass)
    constexpr int M = CHI == MMX_CHI_SCALAR ? 1 : (CHI == MMX_CHI_SYM6 ? 6 : 9);
    constexpr unsigned chunk = (unsigned)(P * N * sizeof(float2));
    if (tid < M) prefetch_l2(a.chi + (int64_t)tid * N3 + tile_base, chunk);
    else if (tid < M + C) prefetch_l2(Ecur + fbase + (int64_t)(tid - M) * N3 + tile_base, chunk);
    else if ((OPS & OP_PRO) != 0 && tid < M + 2 * C)
      prefetch_l2(a.src + fbase + (int64_t)(tid - M - C) * N3 + tile_base, chunk);
  }

  // ---------------- load (16-byte accesses: two neighbouring words) ----------------
  // strided: pair = (pl, pl+1) at the same j; contiguous: pair = (j, j+1) of the same pencil
  if constexpr ((OPS & OP_PRO) != 0) {
    constexpr int PAIRS = N * P / 2;
#pragma unroll 2
    for (int e = tid; e < PAIRS; e += THREADS) {
      int j, pl;
      int64_t off;
      if (STRIDED) { pl = (e % (P / 2)) * 2; j = e / (P / 2); off = (int64_t)j * jstride + pl; }
      else { j = (e % (N / 2)) * 2; pl = e / (N / 2); off = (int64_t)pl * pstride_c + j; }
      const int64_t vox = tile_base + off;
      float4 ev[C], sv[C];
#pragma unroll
      for (int c = 0; c < C; ++c) {
        ev[c] = *reinterpret_cast<const float4*>(Ecur + fbase + c * N3 + vox);
        sv[c] = *reinterpret_cast<const float4*>(a.src + fbase + c * N3 + vox);
      }
      float2 t0[C], t1[C];
      if constexpr (CHI == MMX_CHI_SCALAR) {
        const float4 xv = *reinterpret_cast<const float4*>(a.chi + vox);
        const float2 x0 = cc.a * make_float2(xv.x, xv.y) + cc.b, x1 = cc.a * make_float2(xv.z, xv.w) + cc.b;
#pragma unroll
        for (int c = 0; c < C; ++c) {
          t0[c] = x0 * make_float2(ev[c].x, ev[c].y) + cc.s * make_float2(sv[c].x, sv[c].y);
          t1[c] = x1 * make_float2(ev[c].z, ev[c].w) + cc.s * make_float2(sv[c].z, sv[c].w);
        }
      } else {
        float2 v0[3], v1[3], o0[3], o1[3];
#pragma unroll
        for (int c = 0; c < 3; ++c) {
          v0[c] = make_float2(ev[c].x, ev[c].y);
          v1[c] = make_float2(ev[c].z, ev[c].w);
        }
        apply_chi2<3, CHI>(a.chi, N3, vox, cc, v0, v1, o0, o1);
#pragma unroll
        for (int c = 0; c < 3; ++c) {
          t0[c] = o0[c] + cc.s * make_float2(sv[c].x, sv[c].y);
          t1[c] = o1[c] + cc.s * make_float2(sv[c].z, sv[c].w);
        }
      }
#pragma unroll
      for (int c = 0; c < C; ++c) {
        if (STRIDED) {
          sm[(c * N + j) * SP + pl] = t0[c];
          sm[(c * N + j) * SP + pl + 1] = t1[c];
        } else {
          sm[(c * N + j) * SP + pl] = t0[c];
          sm[(c * N + j + 1) * SP + pl] = t1[c];
        }
      }
    }
  } else {
    constexpr int PAIRS = ELEMS / 2;
#pragma unroll 4
    for (int e = tid; e < PAIRS; e += THREADS) {
      int j, pl, c;
      int64_t off;
      if (STRIDED) {
        pl = (e % (P / 2)) * 2;
        const int r = e / (P / 2);
        j = r % N;
        c = r / N;
        off = (int64_t)j * jstride + pl;
      } else {
        j = (e % (N / 2)) * 2;
        const int r = e / (N / 2);
        pl = r % P;
        c = r / P;
        off = (int64_t)pl * pstride_c + j;
      }
      const float4 v = *reinterpret_cast<const float4*>(a.T + fbase + c * N3 + tile_base + off);
      if (STRIDED) {
        sm[(c * N + j) * SP + pl] = make_float2(v.x, v.y);
        sm[(c * N + j) * SP + pl + 1] = make_float2(v.z, v.w);
      } else {
        sm[(c * N + j) * SP + pl] = make_float2(v.x, v.y);
        sm[(c * N + j + 1) * SP + pl] = make_float2(v.z, v.w);
      }
    }
  }
  __syncthreads();

  if constexpr ((OPS & OP_FWD) != 0) cfft_tile<R, -1, N, C, P, SP, THREADS>(sm, smtw);
  if constexpr ((OPS & OP_G) != 0) {
    // Green multiply; the pass runs along axis 0 and the tile's pencils carry the other axes' k indices
    __shared__ float sk1[P], sk2[P], sk0[N];
    if (tid < P) {
      const int64_t p = in0 + tid;  // inner index == pencil index for axis 0
      float k1 = 0.f, k2 = 0.f;
      if (a.ndim == 3) {
        const int i1 = (int)(p / a.dims[2]);
        const int i2 = (int)(p - (int64_t)i1 * a.dims[2]);
        k1 = a.kv[1][i1];
        k2 = a.kv[2][i2];
      } else if (a.ndim == 2) {
        k1 = a.kv[1][p];
      }
      sk1[tid] = k1;
      sk2[tid] = k2;
    }
    for (int t = tid; t < N; t += THREADS) sk0[t] = a.kv[0][t];
    __syncthreads();
    const R ar = cc.alpha_re, ai = cc.alpha_im;
    const float2 h = divc(make_float2(0.f, ai), make_float2(ar, ai));
    const float ai2s = ai * ai * a.inv_total, ais = -ai * a.inv_total;
    for (int e = tid; e < N * P; e += THREADS) {
      const int pl = e % P;
      const int j = e / P;
      const float k0 = sk0[j], k1 = sk1[pl], k2 = sk2[pl];
      const float kk2 = k0 * k0 + k1 * k1 + k2 * k2;
      // g / N = -i alpha_i / (|k|^2 - alpha) / N = (alpha_i^2, -alpha_i (|k|^2 - ar)) / |den|^2 / N
      const float dr = kk2 - ar;
      const float inv = 1.f / (dr * dr + ai * ai);
      const float2 g = make_float2(ai2s * inv, ais * dr * inv);
      if constexpr (C == 1) {
        const int idx = j * SP + pl;
        sm[idx] = sm[idx] * g;
      } else {
        float2 F[3], PL[3];
        const float kv[3] = {k0, k1, k2};
#pragma unroll
        for (int c = 0; c < 3; ++c) F[c] = sm[(c * N + j) * SP + pl];
        if (j == 0 && in0 + pl == 0) {
#pragma unroll
          for (int c = 0; c < 3; ++c) PL[c] = c < a.ndim ? F[c] : make_float2(0.f, 0.f);
        } else {
          float2 proj = make_float2(0.f, 0.f);
#pragma unroll
          for (int c = 0; c < 3; ++c)
            if (c < a.ndim) proj += kv[c] * F[c];
          proj = proj * (1.f / kk2);
#pragma unroll
          for (int c = 0; c < 3; ++c) PL[c] = c < a.ndim ? kv[c] * proj : make_float2(0.f, 0.f);
        }
        const float2 hs = h * a.inv_total;
#pragma unroll
        for (int c = 0; c < 3; ++c) sm[(c * N + j) * SP + pl] = g * (F[c] - PL[c]) + hs * PL[c];
      }
    }
    __syncthreads();
  }
  if constexpr ((OPS & OP_INV) != 0) cfft_tile<R, +1, N, C, P, SP, THREADS>(sm, smtw);

  // ---------------- store ----------------
  if constexpr ((OPS & OP_EPI) != 0) {
    double dd2 = 0.0, en2 = 0.0;
    constexpr int PAIRS = N * P / 2;
#pragma unroll 2
    for (int e = tid; e < PAIRS; e += THREADS) {
      int j, pl;
      int64_t off;
      if (STRIDED) { pl = (e % (P / 2)) * 2; j = e / (P / 2); off = (int64_t)j * jstride + pl; }
      else { j = (e % (N / 2)) * 2; pl = e / (N / 2); off = (int64_t)pl * pstride_c + j; }
      const int64_t vox = tile_base + off;
      float2 e0[C], e1[C], v0[C], v1[C], d0[C], d1[C];
#pragma unroll
      for (int c = 0; c < C; ++c) {
        const float4 ev = *reinterpret_cast<const float4*>(Ecur + fbase + c * N3 + vox);
        e0[c] = make_float2(ev.x, ev.y);
        e1[c] = make_float2(ev.z, ev.w);
        float2 s0, s1;
        if (STRIDED) { s0 = sm[(c * N + j) * SP + pl]; s1 = sm[(c * N + j) * SP + pl + 1]; }
        else { s0 = sm[(c * N + j) * SP + pl]; s1 = sm[(c * N + j + 1) * SP + pl]; }
        v0[c] = s0 - e0[c];
        v1[c] = s1 - e1[c];
      }
      apply_chi2<C, CHI>(a.chi, N3, vox, cc, v0, v1, d0, d1);
#pragma unroll
      for (int c = 0; c < C; ++c) {
        const float2 n0 = e0[c] + d0[c], n1 = e1[c] + d1[c];
        *reinterpret_cast<float4*>(Eoth + fbase + c * N3 + vox) = make_float4(n0.x, n0.y, n1.x, n1.y);
        dd2 += norm2d(d0[c]) + norm2d(d1[c]);
        en2 += norm2d(n0) + norm2d(n1);
      }
    }
    finish_pass_norms(a, b, dd2, en2);
  } else {
    constexpr int PAIRS = ELEMS / 2;
#pragma unroll 4
    for (int e = tid; e < PAIRS; e += THREADS) {
      int j, pl, c;
      int64_t off;
      float2 v0, v1;
      if (STRIDED) {
        pl = (e % (P / 2)) * 2;
        const int r = e / (P / 2);
        j = r % N;
        c = r / N;
        off = (int64_t)j * jstride + pl;
        v0 = sm[(c * N + j) * SP + pl];
        v1 = sm[(c * N + j) * SP + pl + 1];
      } else {
        j = (e % (N / 2)) * 2;
        const int r = e / (N / 2);
        pl = r % P;
        c = r / P;
        off = (int64_t)pl * pstride_c + j;
        v0 = sm[(c * N + j) * SP + pl];
        v1 = sm[(c * N + j + 1) * SP + pl];
      }
      *reinterpret_cast<float4*>(a.T + fbase + c * N3 + tile_base + off) = make_float4(v0.x, v0.y, v1.x, v1.y);
    }
  }
}
