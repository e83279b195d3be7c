// Device kernels of the split-Richardson iteration: fused FFT passes, the per-RHS accept/reject decision, norms
// and pointwise helpers.
//
// One iteration d = chi [G (chi E + s') - E] (reference solver.py:1070-1075) is executed as one FFT pass per grid
// axis and direction, each pass reading and writing every word once:
//   1D: [PRO FWD G INV EPI]                         (one kernel)
//   2D: [PRO FWD ax1] [FWD G INV ax0] [INV EPI ax1]
//   3D: [PRO FWD ax2] [FWD ax1] [FWD G INV ax0] [INV ax1] [INV EPI ax2]
// PRO = prologue T = chi E + s' on the load of the first pass; G = the Green multiply between the forward and the
// inverse transform of axis 0 (all other axes are already in k-space there); EPI = epilogue of the last pass:
// d = chi (T - E), E_new = E + d written to the other field buffer, with per-CTA partial sums of |d|^2 and |E_new|^2
// reduced in a fixed order by the last tile of each right-hand side, which then takes the accept/reject decision.
#pragma once
#include "../../include/macromax_b200.h"
#include "mmx_fft.cuh"

enum : int {
  OP_PRO = 1,      // prologue: T = chi(alpha) E + s'(alpha)
  OP_FWD = 2,      // forward FFT along the pass axis
  OP_G = 4,        // Green multiply (axis-0 pass only)
  OP_INV = 8,      // inverse FFT along the pass axis
  OP_EPI = 16,     // iteration epilogue: d = chi (T - E); E' = E + d; partial norms
  OP_GINV = 32,    // with OP_G: apply G^{-1} instead of G
  OP_XLOAD = 64,   // first pass of the defect: load x instead of T
  OP_DEFECT = 128  // defect epilogue: s_out = s' + chi x - T, stored as complex64
};

template <class R> struct IterArgs {
  FFTAxis ax;
  int64_t outer, inner;  // pencil geometry of the pass axis (per component, per RHS)
  int P, sP;             // pencils per tile, shared-memory row pitch
  int64_t N;             // voxels per component
  int ndim;
  int dims[3];
  const R* kv[3];        // k-vector tables per axis
  cpx<R>* T;             // work [B][C][N]
  cpx<R>* E0;            // field buffers [B][C][N] (E0 is x for the defect)
  cpx<R>* E1;
  const cpx<R>* chi;     // [m][N]
  const cpx<R>* src;     // [B][C][N]
  const mmx_rhs_state* st;
  double* partials;      // [B][gridDim.x][2]
  unsigned int* done;    // [B] tiles of the epilogue pass finished (reset by the last one)
  R inv_total;           // 1 / N
  float2* aux;           // defect output [B][C][N] complex64
  size_t l2_window;      // bytes of T kept L2-resident (0: off); host-side launch attribute only
  int nrhs;              // number of right-hand sides (persistent passes)
  int poll_limit;        // polls of a staged-input wait before the pass falls back to global loads (k_pipe_pass)
  int csplit;            // > 1: a one-component strided pass over the csplit components of each RHS, which
                         //      blockIdx.y enumerates (RHS-major); 0 or 1: blockIdx.y is the RHS
};

// Programmatic dependent launch.  The pass kernels are launched so that the next pass's CTAs may become resident
// while this grid drains; each pass calls pdl_wait() before it reads anything an earlier kernel writes (the fields,
// the work buffer, the right-hand-side state), which returns once those grids have completed and their memory is
// visible.  pdl_trigger() lets the dependent grid be scheduled as soon as every CTA of this grid has started.
// Both are no-ops for a kernel launched without the attribute.
__device__ __forceinline__ void pdl_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }
__device__ __forceinline__ void pdl_trigger() { asm volatile("griddepcontrol.launch_dependents;" ::: "memory"); }

// |z|^2 accumulated in FP64 (the squares of complex64 words are exact in double)
__device__ __forceinline__ double norm2d(float2 z) { return (double)z.x * z.x + (double)z.y * z.y; }
__device__ __forceinline__ double norm2d(double2 z) { return z.x * z.x + z.y * z.y; }

template <class R> struct ChiCoef {
  cpx<R> a;   // chi(alpha) = a chi0 + b I
  cpx<R> b;
  R s;        // s'(alpha) = s s'0
  R alpha_re, alpha_im;
};

// Component c of this right-hand side's normalised source is identically zero (bit c of reserved[1], set by the
// caller that wrote the source; 0 claims nothing): the prologue may skip reading it.
__device__ __forceinline__ bool source_is_zero(const mmx_rhs_state* st, int c) { return (st->reserved[1] >> c) & 1; }

template <class R> __device__ __forceinline__ ChiCoef<R> chi_coef(const mmx_rhs_state* st) {
  // chi(alpha) = chi0 alpha0_i / alpha_i + i (alpha0 - alpha) / alpha_i ; s'(alpha) = s'0 alpha0_i / alpha_i
  const double ai = st->alpha_im, ar = st->alpha_re;
  const double ratio = st->alpha0_im / ai;
  ChiCoef<R> c;
  c.a = mkc<R>((R)ratio, (R)0);
  // i (d_re + i d_im) / ai = (-d_im + i d_re) / ai
  const double dre = st->alpha0_re - ar, dim = st->alpha0_im - ai;
  c.b = mkc<R>((R)(-dim / ai), (R)(dre / ai));
  c.s = (R)ratio;
  c.alpha_re = (R)ar;
  c.alpha_im = (R)ai;
  return c;
}

__device__ __forceinline__ int64_t pencil_base(int64_t p, int64_t inner, int n) {
  const int64_t o = p / inner;
  return o * (int64_t)n * inner + (p - o * inner);
}

// bulk prefetch of a contiguous global range into L2 (16-byte aligned address, size a multiple of 16)
__device__ __forceinline__ void prefetch_l2(const void* p, unsigned bytes) {
  asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"(p), "r"(bytes) : "memory");
}

// chi(alpha) applied to the C-vector v at voxel vox: out_r = sum_s (a chi_rs + b delta_rs) v_s
template <class R, int C, int CHI>
__device__ __forceinline__ void apply_chi(const cpx<R>* __restrict__ chi, int64_t N, int64_t vox, const ChiCoef<R>& cc,
                                          const cpx<R>* v, cpx<R>* out) {
  if constexpr (CHI == MMX_CHI_SCALAR) {
    const cpx<R> x = cc.a * chi[vox] + cc.b;
#pragma unroll
    for (int c = 0; c < C; ++c) out[c] = x * v[c];
  } else if constexpr (CHI == MMX_CHI_SYM6) {
    // the six distinct entries are read once each (row-major position -> stored entry)
    constexpr int K[9] = {0, 1, 2, 1, 3, 4, 2, 4, 5};
    cpx<R> m[6];
#pragma unroll
    for (int k = 0; k < 6; ++k) m[k] = cc.a * chi[k * N + vox];
#pragma unroll
    for (int r = 0; r < 3; ++r) {
      cpx<R> acc = cc.b * v[r];
#pragma unroll
      for (int s = 0; s < 3; ++s) acc += m[K[r * 3 + s]] * v[s];
      out[r] = acc;
    }
  } else {
#pragma unroll
    for (int r = 0; r < 3; ++r) {
      cpx<R> acc = cc.b * v[r];
#pragma unroll
      for (int s = 0; s < 3; ++s) acc += (cc.a * chi[(r * 3 + s) * N + vox]) * v[s];
      out[r] = acc;
    }
  }
}

template <class R>
__device__ __forceinline__ void block_reduce_2(double x, double y, double* out2) {
  __shared__ double red[2][32];
  const unsigned full = 0xffffffffu;
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    x += __shfl_down_sync(full, x, o);
    y += __shfl_down_sync(full, y, o);
  }
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  if (lane == 0) {
    red[0][warp] = x;
    red[1][warp] = y;
  }
  __syncthreads();
  if (warp == 0) {
    const int nw = (blockDim.x + 31) >> 5;
    x = lane < nw ? red[0][lane] : 0.0;
    y = lane < nw ? red[1][lane] : 0.0;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      x += __shfl_down_sync(full, x, o);
      y += __shfl_down_sync(full, y, o);
    }
    if (lane == 0) {
      out2[0] = x;
      out2[1] = y;
    }
  }
}

// apply_chi at the neighbouring voxels vox and vox + 1 (vox even, N even), complex64: each stored chi entry of the
// two voxels is one 16-byte load
template <int C, int CHI>
__device__ __forceinline__ void apply_chi2(const float2* __restrict__ chi, int64_t N, int64_t vox,
                                           const ChiCoef<float>& cc, const float2* v0, const float2* v1, float2* o0,
                                           float2* o1) {
  constexpr int M = CHI == MMX_CHI_SCALAR ? 1 : (CHI == MMX_CHI_SYM6 ? 6 : 9);
  float2 m0[M], m1[M];
#pragma unroll
  for (int k = 0; k < M; ++k) {
    const float4 w = *reinterpret_cast<const float4*>(chi + k * N + vox);
    m0[k] = cc.a * make_float2(w.x, w.y);
    m1[k] = cc.a * make_float2(w.z, w.w);
  }
  if constexpr (CHI == MMX_CHI_SCALAR) {
    const float2 x0 = m0[0] + cc.b, x1 = m1[0] + cc.b;
#pragma unroll
    for (int c = 0; c < C; ++c) {
      o0[c] = x0 * v0[c];
      o1[c] = x1 * v1[c];
    }
  } else {
    constexpr int K6[9] = {0, 1, 2, 1, 3, 4, 2, 4, 5};
#pragma unroll
    for (int r = 0; r < 3; ++r) {
      float2 a0 = cc.b * v0[r], a1 = cc.b * v1[r];
#pragma unroll
      for (int s = 0; s < 3; ++s) {
        const int k = CHI == MMX_CHI_SYM6 ? K6[r * 3 + s] : r * 3 + s;
        a0 += m0[k] * v0[s];
        a1 += m1[k] * v1[s];
      }
      o0[r] = a0;
      o1[r] = a1;
    }
  }
}

template <class R, int C, bool GINV>
__device__ __forceinline__ void green_step(cpx<R>* sm, const IterArgs<R>& a, int64_t p0, int64_t np_total,
                                           const ChiCoef<R>& cc) {
  const int n = a.ax.n, P = a.P, sP = a.sP;
  const R ar = cc.alpha_re, ai = cc.alpha_im;
  // h = i alpha_i / alpha (longitudinal factor, solver.py:575)
  const cpx<R> h = divc(mkc<R>((R)0, ai), mkc<R>(ar, ai));
  for (int e = threadIdx.x; e < n * P; e += blockDim.x) {
    const int pl = e % P;
    const int j = e / P;
    const int64_t p = p0 + pl;
    if (p >= np_total) continue;
    R k[3] = {(R)0, (R)0, (R)0};
    k[0] = a.kv[0][j];
    if (a.ndim == 3) {
      const int i1 = (int)(p / a.dims[2]);
      const int i2 = (int)(p - (int64_t)i1 * a.dims[2]);
      k[1] = a.kv[1][i1];
      k[2] = a.kv[2][i2];
    } else if (a.ndim == 2) {
      k[1] = a.kv[1][p];
    }
    const R k2 = k[0] * k[0] + k[1] * k[1] + k[2] * k[2];
    // g = -i alpha_i / (|k|^2 - alpha)  (solver.py:566-568)
    const cpx<R> den = mkc<R>(k2 - ar, -ai);
    const cpx<R> g = divc(mkc<R>((R)0, -ai), den);
    if constexpr (C == 1) {
      const int idx = j * sP + pl;
      if constexpr (GINV) sm[idx] = divc(sm[idx], g) * a.inv_total;
      else sm[idx] = sm[idx] * (g * a.inv_total);
    } else {
      cpx<R> F[3], PL[3];
#pragma unroll
      for (int c = 0; c < 3; ++c) F[c] = sm[(c * n + j) * sP + pl];
      const bool origin = (j == 0) && (p == 0);
      if (origin) {
#pragma unroll
        for (int c = 0; c < 3; ++c) PL[c] = c < a.ndim ? F[c] : mkc<R>((R)0, (R)0);
      } else {
        cpx<R> proj = mkc<R>((R)0, (R)0);
#pragma unroll
        for (int c = 0; c < 3; ++c)
          if (c < a.ndim) proj += k[c] * F[c];
        proj = proj * ((R)1 / k2);
#pragma unroll
        for (int c = 0; c < 3; ++c) PL[c] = c < a.ndim ? k[c] * proj : mkc<R>((R)0, (R)0);
      }
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        cpx<R> r;
        if constexpr (GINV) r = divc(F[c] - PL[c], g) + divc(PL[c], h);
        else r = g * (F[c] - PL[c]) + h * PL[c];
        sm[(c * n + j) * sP + pl] = r * a.inv_total;
      }
    }
  }
  __syncthreads();
}

template <class R, int C, int CHI, int OPS>
__global__ void __launch_bounds__(512, 2) k_iter_pass(IterArgs<R> a) {
  extern __shared__ __align__(16) unsigned char mmx_smem_raw[];
  cpx<R>* sm = reinterpret_cast<cpx<R>*>(mmx_smem_raw);
  const int b = blockIdx.y;
  const mmx_rhs_state* st = a.st + b;
  if (!st->active) return;  // convergence mask: uniform over the block
  const ChiCoef<R> cc = chi_coef<R>(st);
  const int n = a.ax.n, P = a.P, sP = a.sP;
  const int64_t N = a.N, inner = a.inner;
  const int64_t np_total = a.outer * inner;
  const int64_t p0 = (int64_t)blockIdx.x * P;
  const int64_t fbase = (int64_t)b * C * N;
  const bool contig = (inner == 1);
  const int cur = st->cur;
  cpx<R>* __restrict__ Ecur = cur ? a.E1 : a.E0;
  cpx<R>* __restrict__ Eoth = cur ? a.E0 : a.E1;

  // ---------------- load ----------------
  if constexpr ((OPS & OP_PRO) != 0) {
#pragma unroll 4
    for (int e = threadIdx.x; e < n * P; e += blockDim.x) {
      int j, pl;
      if (contig) { j = e % n; pl = e / n; } else { pl = e % P; j = e / P; }
      const int64_t p = p0 + pl;
      cpx<R> t[C];
      if (p < np_total) {
        const int64_t vox = pencil_base(p, inner, n) + (int64_t)j * inner;
        cpx<R> v[C];
#pragma unroll
        for (int c = 0; c < C; ++c) v[c] = Ecur[fbase + c * N + vox];
        apply_chi<R, C, CHI>(a.chi, N, vox, cc, v, t);
#pragma unroll
        for (int c = 0; c < C; ++c) t[c] += cc.s * a.src[fbase + c * N + vox];
      } else {
#pragma unroll
        for (int c = 0; c < C; ++c) t[c] = mkc<R>((R)0, (R)0);
      }
#pragma unroll
      for (int c = 0; c < C; ++c) sm[(c * n + j) * sP + pl] = t[c];
    }
  } else {
    const cpx<R>* __restrict__ srcp = ((OPS & OP_XLOAD) != 0) ? a.E0 : a.T;
#pragma unroll 8
    for (int e = threadIdx.x; e < C * n * P; e += blockDim.x) {
      int j, pl, c;
      if (contig) { j = e % n; const int r = e / n; pl = r % P; c = r / P; }
      else { pl = e % P; const int r = e / P; j = r % n; c = r / n; }
      const int64_t p = p0 + pl;
      cpx<R> v = mkc<R>((R)0, (R)0);
      if (p < np_total) v = srcp[fbase + c * N + pencil_base(p, inner, n) + (int64_t)j * inner];
      sm[(c * n + j) * sP + pl] = v;
    }
  }
  __syncthreads();

  // ---------------- transforms ----------------
  if constexpr ((OPS & OP_FWD) != 0) fft_tile<R, -1>(sm, C, P, sP, a.ax);
  if constexpr ((OPS & OP_G) != 0) green_step<R, C, (OPS & OP_GINV) != 0>(sm, a, p0, np_total, cc);
  if constexpr ((OPS & OP_INV) != 0) fft_tile<R, +1>(sm, C, P, sP, a.ax);

  // ---------------- store ----------------
  if constexpr ((OPS & OP_EPI) != 0) {
    double dd2 = 0.0, en2 = 0.0;
    for (int e = threadIdx.x; e < n * P; e += blockDim.x) {
      int j, pl;
      if (contig) { j = e % n; pl = e / n; } else { pl = e % P; j = e / P; }
      const int64_t p = p0 + pl;
      if (p >= np_total) continue;
      const int64_t vox = pencil_base(p, inner, n) + (int64_t)j * inner;
      cpx<R> v[C], dd[C];
#pragma unroll
      for (int c = 0; c < C; ++c) {
        const cpx<R> ev = Ecur[fbase + c * N + vox];
        v[c] = sm[(c * n + j) * sP + pl] - ev;  // G(chi E + s') - E
        dd[c] = ev;                              // keep E for the update
      }
      cpx<R> d[C];
      apply_chi<R, C, CHI>(a.chi, N, vox, cc, v, d);
#pragma unroll
      for (int c = 0; c < C; ++c) {
        const cpx<R> en = dd[c] + d[c];
        Eoth[fbase + c * N + vox] = en;
        dd2 += norm2d(d[c]);
        en2 += norm2d(en);
      }
    }
    finish_pass_norms(a, b, dd2, en2);
  } else if constexpr ((OPS & OP_DEFECT) != 0) {
    for (int e = threadIdx.x; e < n * P; e += blockDim.x) {
      int j, pl;
      if (contig) { j = e % n; pl = e / n; } else { pl = e % P; j = e / P; }
      const int64_t p = p0 + pl;
      if (p >= np_total) continue;
      const int64_t vox = pencil_base(p, inner, n) + (int64_t)j * inner;
      cpx<R> x[C], cx[C];
#pragma unroll
      for (int c = 0; c < C; ++c) x[c] = a.E0[fbase + c * N + vox];
      apply_chi<R, C, CHI>(a.chi, N, vox, cc, x, cx);
#pragma unroll
      for (int c = 0; c < C; ++c) {
        // s'(alpha) + chi(alpha) x - G(alpha)^{-1} x, stored normalised to alpha0 like every source (/ s)
        const cpx<R> s = cc.s * a.src[fbase + c * N + vox] + cx[c] - sm[(c * n + j) * sP + pl];
        a.aux[fbase + c * N + vox] = to_c32(s * ((R)1 / cc.s));
      }
    }
  } else {
    for (int e = threadIdx.x; e < C * n * P; e += blockDim.x) {
      int j, pl, c;
      if (contig) { j = e % n; const int r = e / n; pl = r % P; c = r / P; }
      else { pl = e % P; const int r = e / P; j = r % n; c = r / n; }
      const int64_t p = p0 + pl;
      if (p < np_total) a.T[fbase + c * N + pencil_base(p, inner, n) + (int64_t)j * inner] = sm[(c * n + j) * sP + pl];
    }
  }
}

// Accept / reject of Solution.__iter__ (solver.py:1077-1096) and the stop rule of solve (solver.py:81-83,
// 1112-1121) for one right-hand side, from the epilogue pass partials (deterministic fixed-order reduction).
// Executed by one whole block.
__device__ void decide_rhs(mmx_rhs_state* S, const double* __restrict__ pp, int ntiles) {
  // The block is the only one still running when it gets here, so the reduction is on the critical path: every
  // thread issues its loads U at a time into U independent accumulators (a fixed order for a given ntiles and
  // block size, hence deterministic) instead of one dependent load-add chain.
  constexpr int U = 8;
  const double2* __restrict__ p2 = reinterpret_cast<const double2*>(pp);
  const int nt = blockDim.x;
  double sd[U], se[U];
#pragma unroll
  for (int u = 0; u < U; ++u) sd[u] = se[u] = 0.0;
  int i = threadIdx.x;
  for (; i + (U - 1) * nt < ntiles; i += U * nt) {
    double2 v[U];
#pragma unroll
    for (int u = 0; u < U; ++u) v[u] = p2[i + u * nt];
#pragma unroll
    for (int u = 0; u < U; ++u) {
      sd[u] += v[u].x;
      se[u] += v[u].y;
    }
  }
  for (int u = 0; i < ntiles; i += nt, ++u) {
    const double2 v = p2[i];
    sd[u & (U - 1)] += v.x;
    se[u & (U - 1)] += v.y;
  }
  double dd2 = 0.0, en2 = 0.0;
#pragma unroll
  for (int u = 0; u < U; ++u) {
    dd2 += sd[u];
    en2 += se[u];
  }
  double out2[2];
  block_reduce_2<double>(dd2, en2, out2);
  if (threadIdx.x == 0) {
    const double nu = sqrt(out2[0]);
    S->iteration += 1;
    S->last_norm = nu;
    const double prev = S->prev_norm;
    if (prev == 0.0) {  // Python float division by zero in solver.py:1079
      S->status = MMX_STATUS_ZERODIV;
      S->active = 0;
      return;
    }
    const double rel = nu / prev;
    if (rel < 1.0) {
      S->cur ^= 1;
      S->prev_norm = nu;
      S->field_norm = sqrt(out2[1]);
      S->accepted = 1;
    } else {
      S->alpha_im = 1.5 * S->alpha_im;  // solver.py:1092
      S->rejections += 1;
      S->accepted = 0;
    }
    S->residue = S->prev_norm > 0.0 ? S->prev_norm / S->field_norm : 0.0;
    S->active = ((double)S->iteration < S->maxiter) && (S->residue > S->rtol);
  }
}

__global__ void k_decide(mmx_rhs_state* states, const double* __restrict__ partials, int ntiles) {
  mmx_rhs_state* S = states + blockIdx.x;
  if (!S->active) return;
  decide_rhs(S, partials + (int64_t)blockIdx.x * ntiles * 2, ntiles);
}

// End of the epilogue pass for one tile: publish the tile's partial norms; the last tile of the RHS to finish
// (counted with an atomic after a fence, no waiting) reduces them in a fixed order and takes the decision.
template <class R>
__device__ __forceinline__ void finish_pass_norms(const IterArgs<R>& a, int b, double dd2, double en2) {
  __shared__ int s_last;
  double out2[2];
  block_reduce_2<R>(dd2, en2, out2);
  if (threadIdx.x == 0) {
    double* dst = a.partials + ((int64_t)b * gridDim.x + blockIdx.x) * 2;
    dst[0] = out2[0];
    dst[1] = out2[1];
    __threadfence();
    const unsigned int prev = atomicAdd(a.done + b, 1u);
    s_last = (prev == gridDim.x - 1);
  }
  __syncthreads();
  if (s_last) {
    __threadfence();
    decide_rhs(const_cast<mmx_rhs_state*>(a.st) + b, a.partials + (int64_t)b * gridDim.x * 2, gridDim.x);
    if (threadIdx.x == 0) a.done[b] = 0u;
  }
}

// ------------------------------------------------------------------------------------------------------------
// Plain FFT pass (BackEnd.ft / ift): C = 1, batch folded into the outer dimension.
// ------------------------------------------------------------------------------------------------------------
template <class R> struct FFTPassArgs {
  FFTAxis ax;
  int64_t outer, inner;
  int P, sP;
  const cpx<R>* in;
  cpx<R>* out;
  R scale;
};

template <class R, int DIR> __global__ void __launch_bounds__(512, 2) k_fft_pass(FFTPassArgs<R> a) {
  extern __shared__ __align__(16) unsigned char mmx_smem_raw[];
  cpx<R>* sm = reinterpret_cast<cpx<R>*>(mmx_smem_raw);
  const int n = a.ax.n, P = a.P, sP = a.sP;
  const int64_t inner = a.inner, np_total = a.outer * inner;
  const int64_t p0 = (int64_t)blockIdx.x * P;
  const bool contig = inner == 1;
  for (int e = threadIdx.x; e < n * P; e += blockDim.x) {
    int j, pl;
    if (contig) { j = e % n; pl = e / n; } else { pl = e % P; j = e / P; }
    const int64_t p = p0 + pl;
    cpx<R> v = mkc<R>((R)0, (R)0);
    if (p < np_total) v = a.in[pencil_base(p, inner, n) + (int64_t)j * inner];
    sm[j * sP + pl] = v;
  }
  __syncthreads();
  fft_tile<R, DIR>(sm, 1, P, sP, a.ax);
  for (int e = threadIdx.x; e < n * P; e += blockDim.x) {
    int j, pl;
    if (contig) { j = e % n; pl = e / n; } else { pl = e % P; j = e / P; }
    const int64_t p = p0 + pl;
    if (p < np_total) a.out[pencil_base(p, inner, n) + (int64_t)j * inner] = sm[j * sP + pl] * a.scale;
  }
}

// ------------------------------------------------------------------------------------------------------------
// Norms and pointwise kernels
// ------------------------------------------------------------------------------------------------------------
template <class R> __global__ void k_norm_partials(const cpx<R>* __restrict__ x, int64_t n, double* partials) {
  double s = 0.0;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    s += norm2d(x[i]);
  double out2[2];
  block_reduce_2<R>(s, 0.0, out2);
  if (threadIdx.x == 0) partials[blockIdx.x] = out2[0];
}

__global__ void k_norm_final(const double* __restrict__ partials, int np, double* out) {
  double s = 0.0;
  for (int i = threadIdx.x; i < np; i += blockDim.x) s += partials[i];
  double out2[2];
  block_reduce_2<double>(s, 0.0, out2);
  if (threadIdx.x == 0) out[0] = sqrt(out2[0]);
}

__global__ void k_accumulate(double2* __restrict__ x, const float2* __restrict__ d, int64_t n) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    const float2 v = d[i];
    double2 y = x[i];
    y.x += (double)v.x;
    y.y += (double)v.y;
    x[i] = y;
  }
}

template <class R>
__global__ void k_adjoint_grad(const cpx<R>* __restrict__ E, const cpx<R>* __restrict__ nu, cpx<R>* __restrict__ g,
                               int64_t batch, int ncomp, int64_t nvox, R scale) {
  const int64_t total = batch * nvox;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < total; i += (int64_t)gridDim.x * blockDim.x) {
    const int64_t b = i / nvox, v = i - b * nvox;
    cpx<R> acc = mkc<R>((R)0, (R)0);
    for (int c = 0; c < ncomp; ++c) {
      const int64_t idx = (b * ncomp + c) * nvox + v;
      acc += nu[idx] * E[idx];
    }
    g[i] = conjc(acc) * scale;
  }
}

template <class R>
__global__ void k_pointwise_mul(const cpx<R>* __restrict__ A, int ra, int ca, const cpx<R>* __restrict__ B, int cb,
                                int bstride, cpx<R>* __restrict__ out, int64_t nvox) {
  for (int64_t v = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; v < nvox; v += (int64_t)gridDim.x * blockDim.x) {
    for (int r = 0; r < ra; ++r)
      for (int q = 0; q < cb; ++q) {
        cpx<R> acc = mkc<R>((R)0, (R)0);
        for (int s = 0; s < ca; ++s) acc += A[(r * ca + s) * nvox + v] * B[(s * cb + q) * (bstride ? nvox : 1) + (bstride ? v : 0)];
        out[(r * cb + q) * nvox + v] = acc;
      }
  }
}

// ------------------------------------------------------------------------------------------------------------
// Set-up reductions over 3x3 permittivity fields (FP64): the largest eigenvalue of (ab I - M)^H (ab I - M) for the
// alpha objective (solver.py:392-401) and the extreme eigenvalues of the anti-Hermitian part -0.5i (M - M^H) for the
// gain / loss checks (solver.py:322-336).  Eigenvalues of a Hermitian 3x3 matrix in closed form: trigonometric
// solution of the characteristic cubic, q = tr/3, p = sqrt(tr((H - qI)^2)/6), r = det((H - qI)/p)/2,
// lambda_k = q + 2p cos(acos(r)/3 + 2 pi k/3).
// ------------------------------------------------------------------------------------------------------------
__device__ __forceinline__ void herm3_extremes(const double h[3][3][2], double* lmin, double* lmax) {
  // h[i][j] = (re, im), Hermitian: real diagonal, h[j][i] = conj(h[i][j])
  const double q = (h[0][0][0] + h[1][1][0] + h[2][2][0]) / 3.0;
  const double p1 = h[0][1][0] * h[0][1][0] + h[0][1][1] * h[0][1][1] + h[0][2][0] * h[0][2][0] +
                    h[0][2][1] * h[0][2][1] + h[1][2][0] * h[1][2][0] + h[1][2][1] * h[1][2][1];
  const double d0 = h[0][0][0] - q, d1 = h[1][1][0] - q, d2 = h[2][2][0] - q;
  const double p2 = d0 * d0 + d1 * d1 + d2 * d2 + 2.0 * p1;
  if (p2 <= 0.0) {
    *lmin = q;
    *lmax = q;
    return;
  }
  const double p = sqrt(p2 / 6.0);
  const double ip = 1.0 / p;
  const double b00 = d0 * ip, b11 = d1 * ip, b22 = d2 * ip;
  const double b01r = h[0][1][0] * ip, b01i = h[0][1][1] * ip;
  const double b02r = h[0][2][0] * ip, b02i = h[0][2][1] * ip;
  const double b12r = h[1][2][0] * ip, b12i = h[1][2][1] * ip;
  // det B = b00 b11 b22 + 2 Re(b01 b12 conj(b02)) - b00 |b12|^2 - b11 |b02|^2 - b22 |b01|^2
  const double re_t = (b01r * b12r - b01i * b12i) * b02r + (b01r * b12i + b01i * b12r) * b02i;
  double r = 0.5 * (b00 * b11 * b22 + 2.0 * re_t - b00 * (b12r * b12r + b12i * b12i) -
                    b11 * (b02r * b02r + b02i * b02i) - b22 * (b01r * b01r + b01i * b01i));
  r = fmin(1.0, fmax(-1.0, r));
  const double phi = acos(r) / 3.0;
  *lmax = q + 2.0 * p * cos(phi);
  *lmin = q + 2.0 * p * cos(phi + 2.0943951023931954923);  // + 2 pi / 3
}

// mode 0: out = max_v lambda_max((ab I - M_v)^H (ab I - M_v)); mode 1: out = (min_v, max_v) of the eigenvalues of
// -0.5i (M_v - M_v^H).  M: [9][N] complex128.  Block partials in part[2 * block].
__global__ void k_mat3_extremes(const double2* __restrict__ M, int64_t N, int mode, double ab, double* part) {
  double vmin = INFINITY, vmax = -INFINITY;
  for (int64_t v = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; v < N; v += (int64_t)gridDim.x * blockDim.x) {
    double a[3][3][2];
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
      for (int j = 0; j < 3; ++j) {
        const double2 z = M[(int64_t)(i * 3 + j) * N + v];
        a[i][j][0] = z.x;
        a[i][j][1] = z.y;
      }
    double h[3][3][2];
    if (mode == 0) {
      // D = ab I - M; H = D^H D
      double d[3][3][2];
#pragma unroll
      for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = 0; j < 3; ++j) {
          d[i][j][0] = (i == j ? ab : 0.0) - a[i][j][0];
          d[i][j][1] = -a[i][j][1];
        }
#pragma unroll
      for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = 0; j < 3; ++j) {
          double re = 0.0, im = 0.0;
#pragma unroll
          for (int k = 0; k < 3; ++k) {  // conj(d[k][i]) * d[k][j]
            re += d[k][i][0] * d[k][j][0] + d[k][i][1] * d[k][j][1];
            im += d[k][i][0] * d[k][j][1] - d[k][i][1] * d[k][j][0];
          }
          h[i][j][0] = re;
          h[i][j][1] = im;
        }
    } else {
      // -0.5i (M - M^H) (solver.py:324): entry -(i/2)(m_ij - conj(m_ji)); diagonal = Im m_ii
#pragma unroll
      for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = 0; j < 3; ++j) {
          const double xr = a[i][j][0] - a[j][i][0], xi = a[i][j][1] + a[j][i][1];
          h[i][j][0] = 0.5 * xi;
          h[i][j][1] = -0.5 * xr;
        }
    }
    double lo, hi;
    herm3_extremes(h, &lo, &hi);
    vmin = fmin(vmin, lo);
    vmax = fmax(vmax, hi);
  }
  // block min / max
  __shared__ double smin[32], smax[32];
  const unsigned full = 0xffffffffu;
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    vmin = fmin(vmin, __shfl_down_sync(full, vmin, o));
    vmax = fmax(vmax, __shfl_down_sync(full, vmax, o));
  }
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  if (lane == 0) {
    smin[warp] = vmin;
    smax[warp] = vmax;
  }
  __syncthreads();
  if (warp == 0) {
    const int nw = (blockDim.x + 31) >> 5;
    vmin = lane < nw ? smin[lane] : INFINITY;
    vmax = lane < nw ? smax[lane] : -INFINITY;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      vmin = fmin(vmin, __shfl_down_sync(full, vmin, o));
      vmax = fmax(vmax, __shfl_down_sync(full, vmax, o));
    }
    if (lane == 0) {
      part[2 * blockIdx.x] = vmin;
      part[2 * blockIdx.x + 1] = vmax;
    }
  }
}

// Objective of the alpha search for a scalar permittivity (solver.py:392-401, non-magnetic): the host expression
// |ab|^2 - (conj(eps) ab + eps conj(ab)) + conj(eps) eps has, for real ab, an imaginary part that is exactly zero and
// the real part (ab^2 - 2 round(x ab)) + p with x = Re eps and p = the host's value of Re(conj(eps) eps).  Evaluated
// here with explicitly rounded FP64 operations (no fused multiply-add), so min / max over the voxels are those of
// the host expression bit for bit.  xp: [N] pairs (x, p).  Per-block (min, max) partials as k_mat3_extremes.
// chi = s eps - d I per voxel (m = 1 or 9 row-major entries), from complex128 to the precision of OUT
template <class OUT>
__global__ void k_chi_from_eps(const double2* __restrict__ eps, int m, int64_t N, double2 s, double2 d,
                               OUT* __restrict__ chi) {
  const int64_t total = (int64_t)m * N;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < total; i += (int64_t)gridDim.x * blockDim.x) {
    const int r = (int)(i / N);
    const double2 e = eps[i];
    double2 c = make_double2(s.x * e.x - s.y * e.y, s.x * e.y + s.y * e.x);
    if (m == 1 || r == 0 || r == 4 || r == 8) {
      c.x -= d.x;
      c.y -= d.y;
    }
    if constexpr (std::is_same<OUT, float2>::value) {
      chi[i] = make_float2((float)c.x, (float)c.y);
    } else {
      chi[i] = c;
    }
  }
}

__global__ void k_scalar_sigma(const double2* __restrict__ xp, int64_t N, double ab, double* part) {
  double vmin = INFINITY, vmax = -INFINITY;
  const double ab2 = __dmul_rn(ab, ab);
  for (int64_t v = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; v < N; v += (int64_t)gridDim.x * blockDim.x) {
    const double2 q = xp[v];
    const double t = __dmul_rn(q.x, ab);
    const double w = __dadd_rn(__dsub_rn(ab2, __dadd_rn(t, t)), q.y);
    vmin = fmin(vmin, w);
    vmax = fmax(vmax, w);
  }
  __shared__ double smin[32], smax[32];
  const unsigned full = 0xffffffffu;
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    vmin = fmin(vmin, __shfl_down_sync(full, vmin, o));
    vmax = fmax(vmax, __shfl_down_sync(full, vmax, o));
  }
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  if (lane == 0) {
    smin[warp] = vmin;
    smax[warp] = vmax;
  }
  __syncthreads();
  if (warp == 0) {
    const int nw = (blockDim.x + 31) >> 5;
    vmin = lane < nw ? smin[lane] : INFINITY;
    vmax = lane < nw ? smax[lane] : -INFINITY;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      vmin = fmin(vmin, __shfl_down_sync(full, vmin, o));
      vmax = fmax(vmax, __shfl_down_sync(full, vmax, o));
    }
    if (lane == 0) {
      part[2 * blockIdx.x] = vmin;
      part[2 * blockIdx.x + 1] = vmax;
    }
  }
}

__global__ void k_minmax_final(const double* __restrict__ part, int np, double* out) {
  double vmin = INFINITY, vmax = -INFINITY;
  for (int i = threadIdx.x; i < np; i += blockDim.x) {
    vmin = fmin(vmin, part[2 * i]);
    vmax = fmax(vmax, part[2 * i + 1]);
  }
  __shared__ double smin[32], smax[32];
  const unsigned full = 0xffffffffu;
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    vmin = fmin(vmin, __shfl_down_sync(full, vmin, o));
    vmax = fmax(vmax, __shfl_down_sync(full, vmax, o));
  }
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  if (lane == 0) {
    smin[warp] = vmin;
    smax[warp] = vmax;
  }
  __syncthreads();
  if (warp == 0) {
    const int nw = (blockDim.x + 31) >> 5;
    vmin = lane < nw ? smin[lane] : INFINITY;
    vmax = lane < nw ? smax[lane] : -INFINITY;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      vmin = fmin(vmin, __shfl_down_sync(full, vmin, o));
      vmax = fmax(vmax, __shfl_down_sync(full, vmax, o));
    }
    if (lane == 0) {
      out[0] = vmin;
      out[1] = vmax;
    }
  }
}
