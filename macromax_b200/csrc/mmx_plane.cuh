// Plane passes for 3D grids whose two inner axes are both 128 samples long (complex64, isotropic chi).
//
// The 3D iteration schedule [PRO FWD ax2] [FWD ax1] [FWD G INV ax0] [INV ax1] [INV EPI ax2] keeps the work buffer
// T in L2 through its three middle passes, but every pass still streams T through L2 and pays a launch's worth of
// fill and drain.  The plane passes below do the two inner axes of one (RHS, component, i0) plane in one kernel, so
// an iteration is the 3-sweep schedule itself:
//   k_plane_pass<C, PRO|FWD>:  T = FFT_ax1 FFT_ax2 (chi E + s')            (prologue, forward along axes 2 and 1)
//   k_reg_pass<C, FWD|G|INV>:  the axis-0 pass with the Green multiply (unchanged)
//   k_plane_pass<C, INV|EPI>:  E' = E + chi (IFFT_ax2 IFFT_ax1 T - E)      (inverse along axes 1 and 2, epilogue)
//
// A 128 x 128 plane of complex64 is 128 KB, so one plane is split over a cluster of two CTAs (69 KB of shared
// memory each, three CTAs per SM).  The CTA of cluster rank r holds either the rows [64r, 64r + 64) of the plane
// (row layout, for the axis-2 transforms) or the columns [64r, 64r + 64) (column layout, for the axis-1
// transforms).  In both layouts shared memory is S[64][PITCH]; the row layout stores sample (n, m) of its rows at
// S[n][col(m)], the column layout stores (row R, column j) at S[R mod 64][col(64 (R / 64) + j)], with the skew
// col(m) = m + m / 16 (every strided and unit-stride access below takes the minimum two wavefronts per warp).  The
// two layouts coincide on the quarter S[*][col(64 r + .)]; switching between them swaps the other quarter with the
// peer's through distributed shared memory: read the peer's quarter into registers, cluster barrier, write it.
//
// The length-128 transforms use the radix plan 8 x 16 of the self-sorting formulation in mmx_fft.cuh:
//   stage 1: radix 8, L = 1:  butterfly i < 16 reads x[i + 16 q], writes y[8 i + q]              (q < 8)
//   stage 2: radix 16, L = 8: butterfly i < 8 reads y[i + 8 q], twiddles w^(q i), writes X[i + 8 q] (q < 16)
// The second stage writes its outputs to the positions it read, so it needs no barrier and feeds the epilogue or
// global memory straight from registers.  Each CTA starts with a bulk L2 prefetch of its contiguous input rows
// (cp.async.bulk.prefetch.L2), so that the loads of the first and last stages meet L2 rather than DRAM.
#pragma once
#include <cooperative_groups.h>

#include "mmx_reg.cuh"

namespace mmx_plane {

constexpr int N = 128;           // samples along axes 1 and 2
constexpr int H = 64;            // rows (or columns) per CTA
constexpr int PITCH = N + N / 16;
constexpr int THREADS = 256;
constexpr int RA = 8, TA = N / RA;    // stage 1: radix 8, 16 butterflies per line
constexpr int RB = 16, TB = N / RB;   // stage 2: radix 16, L = 8, 8 butterflies per line

__device__ __forceinline__ int col(int m) { return m + (m >> 4); }
// column layout: logical row R of local column j
__device__ __forceinline__ int cidx(int R, int j) { return (R & (H - 1)) * PITCH + col(((R >> 6) << 6) + j); }
// row layout: local row n, sample m
__device__ __forceinline__ int ridx(int n, int m) { return n * PITCH + col(m); }

inline size_t smem_bytes() { return ((size_t)H * PITCH + N) * sizeof(float2); }

// Swap the off-diagonal quarter with the peer CTA: our S[*][col(64 p + j)] <- peer's S[*][col(64 r + j)].
__device__ __forceinline__ void swap_quarter(float2* sm, cooperative_groups::cluster_group& cluster, int r) {
  const int p = r ^ 1;
  const float2* peer = cluster.map_shared_rank(sm, p);
  constexpr int PER = H * H / THREADS;  // 16 words per thread
  const int j = threadIdx.x % H;
  const int n0 = threadIdx.x / H;       // 0 .. 3
  float2 v[PER];
  cluster.sync();  // the peer's quarter is final
#pragma unroll
  for (int k = 0; k < PER; ++k) v[k] = peer[ridx(n0 + 4 * k, 64 * r + j)];
  cluster.sync();  // the peer has read our quarter before we overwrite it
#pragma unroll
  for (int k = 0; k < PER; ++k) sm[ridx(n0 + 4 * k, 64 * p + j)] = v[k];
  __syncthreads();
}

// Stage 2 (radix 16, L = 8) of butterfly i in registers: on entry v[q] = y[i + 8 q], on return v[q] = X[i + 8 q].
template <int DIR>
__device__ __forceinline__ void stage_b(float2* v, const float2* tw, int i) {
#pragma unroll
  for (int q = 1; q < RB; ++q) {
    float2 w = tw[q * i];
    if (DIR > 0) w = conjc(w);
    v[q] = v[q] * w;
  }
  bfly<float, RB, DIR>(v, tw, N);
}

}  // namespace mmx_plane

// OPS: OP_PRO | OP_FWD (forward plane pass with the prologue) or OP_INV | OP_EPI (inverse plane pass with the
// epilogue).  Grid: (2 n0 C, B) in clusters of 2 along x; cluster c = blockIdx.x / 2 covers plane i0 = c / C of
// component c % C, so the C component planes that share chi's plane run side by side and chi is read from DRAM once.
template <int C, int OPS>
__global__ void __cluster_dims__(2, 1, 1) __launch_bounds__(mmx_plane::THREADS, 3) k_plane_pass(IterArgs<float> a) {
  using namespace mmx_plane;
  namespace cg = cooperative_groups;
  extern __shared__ __align__(16) unsigned char mmx_smem_raw[];
  float2* sm = reinterpret_cast<float2*>(mmx_smem_raw);
  float2* smtw = sm + H * PITCH;
  cg::cluster_group cluster = cg::this_cluster();
  const int b = blockIdx.y;
  const mmx_rhs_state* st = a.st + b;
  pdl_wait();
  pdl_trigger();
  if (!st->active) return;  // both CTAs of a cluster share b, so both leave
  const int r = (int)cluster.block_rank();
  const int tid = threadIdx.x;
  const int plane = blockIdx.x >> 1;
  const int c = plane % C;
  const int64_t i0 = plane / C;
  const int64_t N3 = a.N;
  const int64_t pbase = i0 * (int64_t)(N * N);            // voxel index of (i0, 0, 0)
  const int64_t fbase = ((int64_t)b * C + c) * N3 + pbase;  // word index of this component plane
  const int cur = st->cur;
  // this CTA's rows of E, s' and chi: one contiguous 64 KB chunk each
  const float2* __restrict__ Erows = (cur ? a.E1 : a.E0) + fbase + H * r * N;
  const float2* __restrict__ xrows = a.chi + pbase + H * r * N;
  if (tid == 0) {
    prefetch_l2(Erows, H * N * sizeof(float2));
    prefetch_l2(xrows, H * N * sizeof(float2));
    if constexpr ((OPS & OP_PRO) != 0) prefetch_l2(a.src + fbase + H * r * N, H * N * sizeof(float2));
  }
  const float2* twg = (const float2*)a.ax.tw;
  for (int t = tid; t < N; t += THREADS) smtw[t] = twg[t];
  const ChiCoef<float> cc = chi_coef<float>(st);
  __syncthreads();

  if constexpr (OPS == (OP_PRO | OP_FWD)) {
    const float2* __restrict__ srows = a.src + fbase + H * r * N;
    // rows, stage 1: x = chi(alpha) E + s'(alpha) on the load (16-byte loads of two adjacent butterflies),
    // radix 8 (L = 1), to shared memory
    {
      const int i = 2 * (tid % 8);
#pragma unroll 1
      for (int k = 0; k < 2; ++k) {
        const int n = tid / 8 + 32 * k;
        float2 u0[RA], u1[RA];
#pragma unroll
        for (int q = 0; q < RA; ++q) {
          const int v = n * N + i + q * TA;
          const float4 e = *reinterpret_cast<const float4*>(Erows + v);
          const float4 s = *reinterpret_cast<const float4*>(srows + v);
          const float4 x = *reinterpret_cast<const float4*>(xrows + v);
          u0[q] = (cc.a * make_float2(x.x, x.y) + cc.b) * make_float2(e.x, e.y) + cc.s * make_float2(s.x, s.y);
          u1[q] = (cc.a * make_float2(x.z, x.w) + cc.b) * make_float2(e.z, e.w) + cc.s * make_float2(s.z, s.w);
        }
        bfly<float, RA, -1>(u0, smtw, N);
        bfly<float, RA, -1>(u1, smtw, N);
#pragma unroll
        for (int q = 0; q < RA; ++q) {
          sm[ridx(n, i * RA + q)] = u0[q];
          sm[ridx(n, (i + 1) * RA + q)] = u1[q];
        }
      }
    }
    __syncthreads();
    // rows, stage 2 (in place)
    {
      const int i = tid % TB;
#pragma unroll 1
      for (int k = 0; k < 2; ++k) {
        const int n = tid / TB + 32 * k;
        float2 v[RB];
#pragma unroll
        for (int q = 0; q < RB; ++q) v[q] = sm[ridx(n, i + q * TB)];
        stage_b<-1>(v, smtw, i);
#pragma unroll
        for (int q = 0; q < RB; ++q) sm[ridx(n, i + q * TB)] = v[q];
      }
    }
    swap_quarter(sm, cluster, r);  // row layout -> column layout
    // columns, stage 1 (radix 8, L = 1), in two rounds of 32 columns, two butterflies per thread and round
    {
      const int i = tid / 32;  // butterflies i and i + 8
#pragma unroll 1
      for (int rd = 0; rd < 2; ++rd) {
        const int j = tid % 32 + 32 * rd;
        float2 u0[RA], u1[RA];
#pragma unroll
        for (int q = 0; q < RA; ++q) {
          u0[q] = sm[cidx(i + q * TA, j)];
          u1[q] = sm[cidx(i + 8 + q * TA, j)];
        }
        bfly<float, RA, -1>(u0, smtw, N);
        bfly<float, RA, -1>(u1, smtw, N);
        __syncthreads();
#pragma unroll
        for (int q = 0; q < RA; ++q) {
          sm[cidx(i * RA + q, j)] = u0[q];
          sm[cidx((i + 8) * RA + q, j)] = u1[q];
        }
        __syncthreads();
      }
    }
    // columns, stage 2 straight to T
    {
      float2* __restrict__ Tp = a.T + fbase + H * r;
      const int j = tid % H;
#pragma unroll 1
      for (int k = 0; k < 2; ++k) {
        const int i = tid / H + 4 * k;
        float2 v[RB];
#pragma unroll
        for (int q = 0; q < RB; ++q) v[q] = sm[cidx(i + q * TB, j)];
        stage_b<-1>(v, smtw, i);
#pragma unroll
        for (int q = 0; q < RB; ++q) Tp[(i + q * TB) * N + j] = v[q];
      }
    }
  } else {
    // columns, stage 1 from T (inverse, radix 8)
    {
      const float2* __restrict__ Tp = a.T + fbase + H * r;
      const int j = tid % H;
#pragma unroll 1
      for (int k = 0; k < 4; ++k) {
        const int i = tid / H + 4 * k;
        float2 u[RA];
#pragma unroll
        for (int q = 0; q < RA; ++q) u[q] = Tp[(i + q * TA) * N + j];
        bfly<float, RA, +1>(u, smtw, N);
#pragma unroll
        for (int q = 0; q < RA; ++q) sm[cidx(i * RA + q, j)] = u[q];
      }
    }
    __syncthreads();
    // columns, stage 2 (in place)
    {
      const int j = tid % H;
#pragma unroll 1
      for (int k = 0; k < 2; ++k) {
        const int i = tid / H + 4 * k;
        float2 v[RB];
#pragma unroll
        for (int q = 0; q < RB; ++q) v[q] = sm[cidx(i + q * TB, j)];
        stage_b<+1>(v, smtw, i);
#pragma unroll
        for (int q = 0; q < RB; ++q) sm[cidx(i + q * TB, j)] = v[q];
      }
    }
    swap_quarter(sm, cluster, r);  // column layout -> row layout
    // rows, stage 1 (radix 8), in two rounds of 32 rows, two butterflies per thread and round
    {
      const int i = tid % TA;
#pragma unroll 1
      for (int rd = 0; rd < 2; ++rd) {
        const int n0 = tid / TA + 32 * rd;  // rows n0 and n0 + 16
        float2 u0[RA], u1[RA];
#pragma unroll
        for (int q = 0; q < RA; ++q) {
          u0[q] = sm[ridx(n0, i + q * TA)];
          u1[q] = sm[ridx(n0 + 16, i + q * TA)];
        }
        bfly<float, RA, +1>(u0, smtw, N);
        bfly<float, RA, +1>(u1, smtw, N);
        __syncthreads();
#pragma unroll
        for (int q = 0; q < RA; ++q) {
          sm[ridx(n0, i * RA + q)] = u0[q];
          sm[ridx(n0 + 16, i * RA + q)] = u1[q];
        }
        __syncthreads();
      }
    }
    // rows, stage 2 and the epilogue d = chi(alpha)(T - E), E' = E + d, with FP64 partial norms
    float2* __restrict__ Eoth = (cur ? a.E0 : a.E1) + fbase + H * r * N;
    double dd2 = 0.0, en2 = 0.0;
    {
      const int i = tid % TB;
#pragma unroll 1
      for (int k = 0; k < 2; ++k) {
        const int n = tid / TB + 32 * k;
        float2 v[RB];
#pragma unroll
        for (int q = 0; q < RB; ++q) v[q] = sm[ridx(n, i + q * TB)];
        stage_b<+1>(v, smtw, i);
#pragma unroll
        for (int q = 0; q < RB; ++q) {
          const int vx = n * N + i + q * TB;
          const float2 e = Erows[vx];
          const float2 d = (cc.a * xrows[vx] + cc.b) * (v[q] - e);
          const float2 en = e + d;
          Eoth[vx] = en;
          dd2 += norm2d(d);
          en2 += norm2d(en);
        }
      }
    }
    finish_pass_norms(a, b, dd2, en2);
  }
}
