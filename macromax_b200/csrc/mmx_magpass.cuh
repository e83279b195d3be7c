// Fused pass schedule of the iteration for magnetic and bi-(an)isotropic media (reference solver.py:531-552,
// 1070-1096), 2D and 3D grids.
//
// The reference's chi_op for these media is chi(x) = chi_EE x + chi_HE D x + D(chi_EH x + chi_HH D x) with the
// spectral curl D = IFFT i k x FFT (backend/__init__.py:472-509), and an iteration is
//   d = chi(G(chi(E) + s') - E),  E += d if ||d|| decreased  (solver.py:1070-1096).
// Here the block products and the spectral operations run inside the FFT passes, one pass per axis and direction
// (axis 0 is the strided outer axis and carries every k-space operation; the last axis is contiguous and carries
// every real-space operation):
//
//   E_FWD    (last axis)  E -> forward                                                      -> A
//   K_CURL_E (axis 0)     forward; FFT(E) kept in Eh; i k x; inverse                        -> A   (D E)
//   MIX1     (last axis)  inverse -> D E; u = chi_EE E + chi_HE D E + s', w = chi_EH E + chi_HH D E;
//                         forward of (u, w)                                                 -> A, B
//   K_GREEN  (axis 0)     forward; Q = FFT(u) + i k x FFT(w) = FFT(chi E + s'); G Q (dyadic Green function with the
//                         reference's DC and missing-axis rules); C = i k x (G Q - FFT(E)); inverse of (G Q, C)
//                                                                                           -> A, B
//   MIX2     (last axis)  inverse -> G(chi E + s'), D t; t = G(...) - E; u2 = chi_EE t + chi_HE D t (kept in U2),
//                         w2 = chi_EH t + chi_HH D t; forward of w2                         -> A
//   K_CURL   (axis 0)     forward; i k x; inverse                                           -> A   (D w2)
//   UPDATE   (last axis)  inverse -> D w2; d = u2 + D w2; E' = E + d into the other field buffer, FP64 partial norms,
//                         the divergence guard and stop rule by the last CTA (decide_rhs)
//
// with the forward and inverse passes of the middle axis (3D) between them (MID_FWD/INV on 3 or 6 components).  The
// four 3x3 blocks are stored once at alpha0 and rescaled to the right-hand side's current alpha on the fly
// (solver.py:514-528: every block by alpha0_i / alpha_i, chi_EE also shifted by i (alpha0 - alpha) / alpha_i; the
// source by alpha0_i / alpha_i).  The 1/N of the inverse transforms is applied with every k-space operation.
// Tiles, shared-memory layout and radix stages are those of k_iter_pass (runtime lengths, mmx_fft.cuh).
#pragma once
#include "mmx_kernels.cuh"

enum MagMode : int {
  MAG_E_FWD = 1,
  MAG_MID_FWD3,
  MAG_MID_INV3,
  MAG_MID_FWD6,
  MAG_MID_INV6,
  MAG_K_CURL_E,
  MAG_K_GREEN,
  MAG_K_CURL,
  MAG_MIX1,
  MAG_MIX2,
  MAG_UPDATE
};

template <class R> struct MagArgs {
  FFTAxis ax;
  int64_t outer, inner;  // pencil geometry of the pass axis
  int P, sP;             // pencils per tile, shared-memory row pitch
  int64_t N;             // voxels
  int ndim;
  int dims[3];
  const R* kv[3];        // k-vector tables (k0-scaled grid)
  R inv_total;           // 1 / N
  cpx<R>* E0;            // field buffers [3][N] (ping-pong, st->cur selects)
  cpx<R>* E1;
  const cpx<R>* src;     // s'0 [3][N]
  const cpx<R>* ee;      // susceptibility blocks at alpha0, [9][N] each
  const cpx<R>* eh;
  const cpx<R>* he;
  const cpx<R>* hh;
  cpx<R>* A;             // work [3][N]
  cpx<R>* B;             // work [3][N] (the second half of 6-component tiles)
  cpx<R>* Eh;            // FFT(E) [3][N]
  cpx<R>* U2;            // u of the second chi application [3][N]
  mmx_rhs_state* st;
  double* partials;      // [gridDim.x][2]
  unsigned int* done;
};

template <int MODE> struct MagModeInfo {
  static constexpr bool six_in = MODE == MAG_MID_FWD6 || MODE == MAG_MID_INV6 || MODE == MAG_K_GREEN ||
                                 MODE == MAG_MIX2;
  static constexpr int C = (six_in || MODE == MAG_MIX1) ? 6 : 3;  // components the tile holds
};

// the block coefficients at the current alpha: f = alpha0_i / alpha_i, chi_EE shift i (alpha0 - alpha) / alpha_i
template <class R> struct MagCoef {
  R f;
  cpx<R> shift;
};
template <class R> __device__ __forceinline__ MagCoef<R> mag_coef(const mmx_rhs_state* st) {
  MagCoef<R> m;
  m.f = (R)(st->alpha0_im / st->alpha_im);
  m.shift = mkc<R>((R)(-(st->alpha0_im - st->alpha_im) / st->alpha_im),
                   (R)((st->alpha0_re - st->alpha_re) / st->alpha_im));
  return m;
}

// u = f (chi_EE0 x + chi_HE0 d) + shift x,  w = f (chi_EH0 x + chi_HH0 d)  at voxel v
template <class R>
__device__ __forceinline__ void mag_mix(const MagArgs<R>& a, const MagCoef<R>& mc, int64_t v, const cpx<R>* x,
                                        const cpx<R>* d, cpx<R>* u, cpx<R>* w) {
  const int64_t N = a.N;
#pragma unroll
  for (int r = 0; r < 3; ++r) {
    cpx<R> ue = mkc<R>((R)0, (R)0), we = ue;
#pragma unroll
    for (int s = 0; s < 3; ++s) {
      const int64_t m = (int64_t)(r * 3 + s) * N + v;
      ue += a.ee[m] * x[s] + a.he[m] * d[s];
      we += a.eh[m] * x[s] + a.hh[m] * d[s];
    }
    u[r] = mc.f * ue + mc.shift * x[r];
    w[r] = mc.f * we;
  }
}

// i k x F
template <class R> __device__ __forceinline__ void curl_k(const R* k, const cpx<R>* F, cpx<R>* out) {
  out[0] = mul_i(k[1] * F[2] - k[2] * F[1], 1);
  out[1] = mul_i(k[2] * F[0] - k[0] * F[2], 1);
  out[2] = mul_i(k[0] * F[1] - k[1] * F[0], 1);
}

template <class R, int MODE>
__global__ void __launch_bounds__(512, 2) k_mag_pass(MagArgs<R> a) {
  using Info = MagModeInfo<MODE>;
  constexpr int C = Info::C;
  extern __shared__ __align__(16) unsigned char mmx_smem_raw[];
  cpx<R>* sm = reinterpret_cast<cpx<R>*>(mmx_smem_raw);
  mmx_rhs_state* st = a.st;
  if (!st->active) return;  // uniform over the grid
  const int n = a.ax.n, P = a.P, sP = a.sP;
  const int64_t N = a.N, inner = a.inner;
  const int64_t np_total = a.outer * inner;
  const int64_t p0 = (int64_t)blockIdx.x * P;
  const bool contig = (inner == 1);
  const int cur = st->cur;
  const cpx<R>* __restrict__ Ecur = cur ? a.E1 : a.E0;
  cpx<R>* __restrict__ Eoth = cur ? a.E0 : a.E1;
  const cpx<R> zero = mkc<R>((R)0, (R)0);
  // loop over the tile's (component, sample, pencil) words in an order that keeps global accesses coalesced
  auto word = [&](int e, int nc, int& c, int& j, int& pl) {
    if (contig) {
      j = e % n;
      const int r = e / n;
      pl = r % P;
      c = r / P;
    } else {
      pl = e % P;
      const int r = e / P;
      j = r % n;
      c = r / n;
    }
    (void)nc;
  };
  auto voxel = [&](int64_t p, int j) { return pencil_base(p, inner, n) + (int64_t)j * inner; };

  // ---------------- load ----------------
  {
    constexpr int CIN = (MODE == MAG_MIX1) ? 3 : C;
    for (int e = threadIdx.x; e < CIN * n * P; e += blockDim.x) {
      int c, j, pl;
      word(e, CIN, c, j, pl);
      const int64_t p = p0 + pl;
      cpx<R> v = zero;
      if (p < np_total) {
        const int64_t vox = voxel(p, j);
        if constexpr (MODE == MAG_E_FWD) v = Ecur[c * N + vox];
        else v = c < 3 ? a.A[c * N + vox] : a.B[(c - 3) * N + vox];
      }
      sm[(c * n + j) * sP + pl] = v;
    }
  }
  __syncthreads();

  // ---------------- first transform ----------------
  if constexpr (MODE == MAG_E_FWD || MODE == MAG_MID_FWD3 || MODE == MAG_K_CURL_E || MODE == MAG_K_CURL)
    fft_tile<R, -1>(sm, 3, P, sP, a.ax);
  if constexpr (MODE == MAG_MID_FWD6 || MODE == MAG_K_GREEN) fft_tile<R, -1>(sm, 6, P, sP, a.ax);
  if constexpr (MODE == MAG_MID_INV3 || MODE == MAG_MIX1 || MODE == MAG_UPDATE) fft_tile<R, +1>(sm, 3, P, sP, a.ax);
  if constexpr (MODE == MAG_MID_INV6 || MODE == MAG_MIX2) fft_tile<R, +1>(sm, 6, P, sP, a.ax);

  // ---------------- per-sample operation ----------------
  if constexpr (MODE == MAG_K_CURL_E || MODE == MAG_K_CURL || MODE == MAG_K_GREEN) {
    // k-space: sample j of axis 0, pencil p over the other axes
    cpx<R> h = zero;
    R ar = (R)0, ai = (R)0;
    if constexpr (MODE == MAG_K_GREEN) {
      ar = (R)st->alpha_re;
      ai = (R)st->alpha_im;
      h = divc(mkc<R>((R)0, ai), mkc<R>(ar, ai));  // i alpha_i / alpha (solver.py:575)
    }
    for (int e = threadIdx.x; e < n * P; e += blockDim.x) {
      const int pl = e % P;
      const int j = e / P;
      const int64_t p = p0 + pl;
      if (p >= np_total) continue;
      R k[3] = {a.kv[0][j], (R)0, (R)0};
      if (a.ndim == 3) {
        const int i1 = (int)(p / a.dims[2]);
        const int i2 = (int)(p - (int64_t)i1 * a.dims[2]);
        k[1] = a.kv[1][i1];
        k[2] = a.kv[2][i2];
      } else {
        k[1] = a.kv[1][p];
      }
      const int64_t vox = voxel(p, j);
      cpx<R> F[3], out[3];
#pragma unroll
      for (int c = 0; c < 3; ++c) F[c] = sm[(c * n + j) * sP + pl];
      if constexpr (MODE == MAG_K_CURL_E || MODE == MAG_K_CURL) {
        if constexpr (MODE == MAG_K_CURL_E) {
#pragma unroll
          for (int c = 0; c < 3; ++c) a.Eh[c * N + vox] = F[c];  // FFT(E), unscaled
        }
        curl_k<R>(k, F, out);
#pragma unroll
        for (int c = 0; c < 3; ++c) sm[(c * n + j) * sP + pl] = out[c] * a.inv_total;
      } else {
        // Q = FFT(u + s') + i k x FFT(w)
        cpx<R> W[3], Q[3];
#pragma unroll
        for (int c = 0; c < 3; ++c) W[c] = sm[((3 + c) * n + j) * sP + pl];
        curl_k<R>(k, W, Q);
#pragma unroll
        for (int c = 0; c < 3; ++c) Q[c] += F[c];
        // G Q = g (Q - P_L Q) + h P_L Q, g = -i alpha_i / (|k|^2 - alpha)  (solver.py:566-577)
        const R k2 = k[0] * k[0] + k[1] * k[1] + k[2] * k[2];
        const cpx<R> g = divc(mkc<R>((R)0, -ai), mkc<R>(k2 - ar, -ai));
        cpx<R> PL[3];
        if (j == 0 && p == 0) {  // DC: P_L Q = Q on the grid's axes (backend/__init__.py:633-644)
#pragma unroll
          for (int c = 0; c < 3; ++c) PL[c] = c < a.ndim ? Q[c] : zero;
        } else {
          cpx<R> proj = zero;
#pragma unroll
          for (int c = 0; c < 3; ++c)
            if (c < a.ndim) proj += k[c] * Q[c];
          proj = proj * ((R)1 / k2);
#pragma unroll
          for (int c = 0; c < 3; ++c) PL[c] = c < a.ndim ? k[c] * proj : zero;
        }
        cpx<R> GQ[3], T[3];
#pragma unroll
        for (int c = 0; c < 3; ++c) {
          GQ[c] = g * (Q[c] - PL[c]) + h * PL[c];
          T[c] = GQ[c] - a.Eh[c * N + vox];  // FFT(t) = FFT(G(chi E + s')) - FFT(E)
        }
        curl_k<R>(k, T, out);
#pragma unroll
        for (int c = 0; c < 3; ++c) {
          sm[(c * n + j) * sP + pl] = GQ[c] * a.inv_total;
          sm[((3 + c) * n + j) * sP + pl] = out[c] * a.inv_total;
        }
      }
    }
    __syncthreads();
  } else if constexpr (MODE == MAG_MIX1 || MODE == MAG_MIX2 || MODE == MAG_UPDATE) {
    // real space: voxel (pencil p, sample j) of the contiguous axis
    const MagCoef<R> mc = mag_coef<R>(st);
    double dd2 = 0.0, en2 = 0.0;
    for (int e = threadIdx.x; e < n * P; e += blockDim.x) {
      const int j = e % n;
      const int pl = e / n;
      const int64_t p = p0 + pl;
      if (p >= np_total) continue;
      const int64_t vox = voxel(p, j);
      cpx<R> x[3], d[3], u[3], w[3];
      if constexpr (MODE == MAG_MIX1) {
#pragma unroll
        for (int c = 0; c < 3; ++c) {
          x[c] = Ecur[c * N + vox];
          d[c] = sm[(c * n + j) * sP + pl];  // D E
        }
        mag_mix<R>(a, mc, vox, x, d, u, w);
#pragma unroll
        for (int c = 0; c < 3; ++c) {
          sm[(c * n + j) * sP + pl] = u[c] + mc.f * a.src[c * N + vox];  // chi_EE E + chi_HE D E + s'(alpha)
          sm[((3 + c) * n + j) * sP + pl] = w[c];
        }
      } else if constexpr (MODE == MAG_MIX2) {
#pragma unroll
        for (int c = 0; c < 3; ++c) {
          x[c] = sm[(c * n + j) * sP + pl] - Ecur[c * N + vox];  // t = G(chi E + s') - E
          d[c] = sm[((3 + c) * n + j) * sP + pl];                 // D t
        }
        mag_mix<R>(a, mc, vox, x, d, u, w);
#pragma unroll
        for (int c = 0; c < 3; ++c) {
          a.U2[c * N + vox] = u[c];
          sm[(c * n + j) * sP + pl] = w[c];
        }
      } else {
#pragma unroll
        for (int c = 0; c < 3; ++c) {
          const cpx<R> dv = a.U2[c * N + vox] + sm[(c * n + j) * sP + pl];  // d = u2 + D w2
          const cpx<R> ev = Ecur[c * N + vox];
          const cpx<R> en = ev + dv;
          Eoth[c * N + vox] = en;
          dd2 += norm2d(dv);
          en2 += norm2d(en);
        }
      }
    }
    if constexpr (MODE == MAG_UPDATE) {
      // per-tile partial norms; the last tile to finish takes the decision (decide_rhs, solver.py:1077-1096)
      __shared__ int s_last;
      double out2[2];
      block_reduce_2<R>(dd2, en2, out2);
      if (threadIdx.x == 0) {
        a.partials[2 * blockIdx.x] = out2[0];
        a.partials[2 * blockIdx.x + 1] = out2[1];
        __threadfence();
        const unsigned int prev = atomicAdd(a.done, 1u);
        s_last = (prev == gridDim.x - 1);
      }
      __syncthreads();
      if (s_last) {
        __threadfence();
        decide_rhs(st, a.partials, gridDim.x);
        if (threadIdx.x == 0) a.done[0] = 0u;
      }
      return;
    }
    __syncthreads();
  }

  // ---------------- second transform ----------------
  if constexpr (MODE == MAG_K_CURL_E || MODE == MAG_K_CURL) fft_tile<R, +1>(sm, 3, P, sP, a.ax);
  if constexpr (MODE == MAG_K_GREEN) fft_tile<R, +1>(sm, 6, P, sP, a.ax);
  if constexpr (MODE == MAG_MIX1) fft_tile<R, -1>(sm, 6, P, sP, a.ax);
  if constexpr (MODE == MAG_MIX2) fft_tile<R, -1>(sm, 3, P, sP, a.ax);

  // ---------------- store ----------------
  constexpr int COUT = (MODE == MAG_MIX2) ? 3 : (MODE == MAG_MIX1 ? 6 : C);
  for (int e = threadIdx.x; e < COUT * n * P; e += blockDim.x) {
    int c, j, pl;
    word(e, COUT, c, j, pl);
    const int64_t p = p0 + pl;
    if (p >= np_total) continue;
    const int64_t vox = voxel(p, j);
    const cpx<R> v = sm[(c * n + j) * sP + pl];
    if (c < 3) a.A[c * N + vox] = v;
    else a.B[(c - 3) * N + vox] = v;
  }
}

// After a chunk of iterations: the current field back in the caller's buffer E0 (mmx_magnetic_iterate updates E in
// place), cur = 0.
template <class R>
__global__ void k_mag_settle(cpx<R>* __restrict__ E0, const cpx<R>* __restrict__ E1, mmx_rhs_state* st, int64_t n) {
  if (st->cur == 0) return;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    E0[i] = E1[i];
}
__global__ void k_mag_settle_state(mmx_rhs_state* st) {
  if (threadIdx.x == 0) st->cur = 0;
}
