// Building blocks of the iteration for magnetic and bi-(an)isotropic media (reference solver.py:531-552).
//
// The magnetic susceptibility operator is chi(x) = chi_EE x + chi_HE D x + D(chi_EH x + chi_HH D x), with D the
// spectral curl i k x (backend/__init__.py:472-509; k of the k0-scaled grid).  It is applied twice per iteration,
// so an iteration costs four curls (FFT pairs) plus the Green function's FFT pair; the host composes it from the
// batched FFT (mmx_fftn) and the pointwise kernels below:
//   k_curl_ft:   F -> i k x F for a 3-component spectrum [3][N] (optionally add + i k x (F - sub))
//   k_green_ft:  the dyadic Green multiply g (F - P_L F) + (i a_i / a) P_L F (reference DC and missing-axis rules)
//   k_chi_mix:   u = chi_EE(alpha) x + chi_HE(alpha) d, w = chi_EH(alpha) x + chi_HH(alpha) d per voxel, with the four
//                3x3 blocks stored once at alpha0 and rescaled on the fly (solver.py:514-528)
//   k_axpby:     out = a x + b y
#pragma once
#include "mmx_kernels.cuh"

struct KGrid {
  int ndim;
  int dims[3];
  int64_t N;
};

template <class R>
__device__ __forceinline__ void k_of_voxel(const KGrid& g, const R* const* kv, int64_t v, R* k) {
  k[0] = k[1] = k[2] = (R)0;
  int64_t rest = v;
  for (int a = g.ndim - 1; a >= 0; --a) {
    const int64_t n = g.dims[a];
    const int64_t i = rest % n;
    rest /= n;
    k[a] = kv[a][i];
  }
}

// out = add + i k x (F - sub); add and sub may be null (then 0); add may be out itself (each voxel is read before
// it is written, by the same thread)
template <class R>
__global__ void k_curl_ft(const cpx<R>* __restrict__ F, cpx<R>* out, KGrid g, const R* kv0, const R* kv1,
                          const R* kv2, const cpx<R>* add = nullptr, const cpx<R>* __restrict__ sub = nullptr) {
  const R* kv[3] = {kv0, kv1, kv2};
  const int64_t N = g.N;
  for (int64_t v = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; v < N; v += (int64_t)gridDim.x * blockDim.x) {
    R k[3];
    k_of_voxel<R>(g, kv, v, k);
    cpx<R> f0 = F[v], f1 = F[N + v], f2 = F[2 * N + v];
    if (sub) {
      f0 -= sub[v];
      f1 -= sub[N + v];
      f2 -= sub[2 * N + v];
    }
    // (k x F)_d = k_{d+1} F_{d-1} - k_{d-1} F_{d+1}; axes beyond the grid have k = 0
    const cpx<R> c0 = k[1] * f2 - k[2] * f1;
    const cpx<R> c1 = k[2] * f0 - k[0] * f2;
    const cpx<R> c2 = k[0] * f1 - k[1] * f0;
    if (add) {
      out[v] = add[v] + mul_i(c0, 1);
      out[N + v] = add[N + v] + mul_i(c1, 1);
      out[2 * N + v] = add[2 * N + v] + mul_i(c2, 1);
    } else {
      out[v] = mul_i(c0, 1);
      out[N + v] = mul_i(c1, 1);
      out[2 * N + v] = mul_i(c2, 1);
    }
  }
}

// st: when not null, alpha is the right-hand side's current alpha (device-resident iteration) instead of (ar, ai)
template <class R>
__global__ void k_green_ft(cpx<R>* __restrict__ F, KGrid g, const R* kv0, const R* kv1, const R* kv2, R ar, R ai,
                           const mmx_rhs_state* st) {
  if (st) {
    ar = (R)st->alpha_re;
    ai = (R)st->alpha_im;
  }
  const R* kv[3] = {kv0, kv1, kv2};
  const int64_t N = g.N;
  const cpx<R> h = divc(mkc<R>((R)0, ai), mkc<R>(ar, ai));  // i alpha_i / alpha (solver.py:575)
  for (int64_t v = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; v < N; v += (int64_t)gridDim.x * blockDim.x) {
    R k[3];
    k_of_voxel<R>(g, kv, v, k);
    const R k2 = k[0] * k[0] + k[1] * k[1] + k[2] * k[2];
    const cpx<R> gs = divc(mkc<R>((R)0, -ai), mkc<R>(k2 - ar, -ai));  // -i alpha_i / (|k|^2 - alpha)
    cpx<R> Fv[3], PL[3];
#pragma unroll
    for (int c = 0; c < 3; ++c) Fv[c] = F[c * N + v];
    if (v == 0) {
#pragma unroll
      for (int c = 0; c < 3; ++c) PL[c] = c < g.ndim ? Fv[c] : mkc<R>((R)0, (R)0);
    } else {
      cpx<R> proj = mkc<R>((R)0, (R)0);
#pragma unroll
      for (int c = 0; c < 3; ++c)
        if (c < g.ndim) proj += k[c] * Fv[c];
      proj = proj * ((R)1 / k2);
#pragma unroll
      for (int c = 0; c < 3; ++c) PL[c] = c < g.ndim ? k[c] * proj : mkc<R>((R)0, (R)0);
    }
#pragma unroll
    for (int c = 0; c < 3; ++c) F[c * N + v] = gs * (Fv[c] - PL[c]) + h * PL[c];
  }
}

// coef: [ee_a, ee_b, eh_f, he_f, hh_f] as complex pairs: chi_EE(alpha) = ee_a chi_EE0 + ee_b I, the others scaled.
// st: when not null, the coefficients follow from the right-hand side's current alpha: f = alpha0_i / alpha_i for
// every block and ee_b = i (alpha0 - alpha) / alpha_i (solver.py:514-528).
template <class R>
__global__ void k_chi_mix(const cpx<R>* __restrict__ x, const cpx<R>* __restrict__ d, const cpx<R>* __restrict__ ee,
                          const cpx<R>* __restrict__ eh, const cpx<R>* __restrict__ he, const cpx<R>* __restrict__ hh,
                          cpx<R> ee_a, cpx<R> ee_b, cpx<R> eh_f, cpx<R> he_f, cpx<R> hh_f, cpx<R>* __restrict__ u,
                          cpx<R>* __restrict__ w, int64_t N, const mmx_rhs_state* st) {
  if (st) {
    const double f = st->alpha0_im / st->alpha_im;
    ee_a = eh_f = he_f = hh_f = mkc<R>((R)f, (R)0);
    // i (alpha0 - alpha) / alpha_i = (-(alpha0_i - alpha_i) + i (alpha0_r - alpha_r)) / alpha_i
    ee_b = mkc<R>((R)(-(st->alpha0_im - st->alpha_im) / st->alpha_im), (R)((st->alpha0_re - st->alpha_re) / st->alpha_im));
  }
  for (int64_t v = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; v < N; v += (int64_t)gridDim.x * blockDim.x) {
    cpx<R> xv[3], dv[3];
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      xv[c] = x[c * N + v];
      dv[c] = d[c * N + v];
    }
#pragma unroll
    for (int r = 0; r < 3; ++r) {
      cpx<R> ue = mkc<R>((R)0, (R)0), uh = mkc<R>((R)0, (R)0), we = mkc<R>((R)0, (R)0), wh = mkc<R>((R)0, (R)0);
#pragma unroll
      for (int s = 0; s < 3; ++s) {
        const int64_t m = (int64_t)(r * 3 + s) * N + v;
        ue += ee[m] * xv[s];
        uh += he[m] * dv[s];
        we += eh[m] * xv[s];
        wh += hh[m] * dv[s];
      }
      u[r * N + v] = ee_a * ue + ee_b * xv[r] + he_f * uh;
      w[r * N + v] = eh_f * we + hh_f * wh;
    }
  }
}

template <class R>
__global__ void k_axpby(cpx<R>* __restrict__ out, const cpx<R>* __restrict__ x, const cpx<R>* __restrict__ y,
                        cpx<R> a, cpx<R> b, int64_t n) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    out[i] = a * x[i] + b * y[i];
}

// ---------------------------------------------------------------------------------------------------------------
// Device-resident iteration (mmx_magnetic_iterate): the accept / reject and stop rules of Solution.__iter__ /
// solve (solver.py:1077-1096, 81-83) on the right-hand side's mmx_rhs_state, so that a chunk of iterations runs
// without the host.  st->reserved[0] is 1 when the current iteration ran (the right-hand side was active at its
// decision), so that its accepted update is still applied when the stop rule then ends the solve.
// ---------------------------------------------------------------------------------------------------------------

// out = u + (alpha0_i / alpha_i) s   (the spatial part of chi E + s'(alpha) whose curl term is added in k-space)
template <class R>
__global__ void k_mag_usrc(cpx<R>* __restrict__ out, const cpx<R>* __restrict__ u, const cpx<R>* __restrict__ src,
                           const mmx_rhs_state* st, int64_t n) {
  const R f = (R)(st->alpha0_im / st->alpha_im);
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    out[i] = u[i] + f * src[i];
}

// d = u + dx, with per-block FP64 partial sums of |d|^2, |E + d|^2 and |E|^2 (partials [gridDim.x][3])
template <class R>
__global__ void k_mag_update(cpx<R>* __restrict__ d, const cpx<R>* __restrict__ u, const cpx<R>* __restrict__ dx,
                             const cpx<R>* __restrict__ E, int64_t n, double* __restrict__ partials) {
  double s0 = 0.0, s1 = 0.0, s2 = 0.0;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    const cpx<R> dv = u[i] + dx[i];
    const cpx<R> e = E[i];
    d[i] = dv;
    s0 += norm2d(dv);
    s1 += norm2d(e + dv);
    s2 += norm2d(e);
  }
  double out2[2];
  block_reduce_2<double>(s0, s1, out2);
  const double t0 = out2[0], t1 = out2[1];
  __syncthreads();
  block_reduce_2<double>(s2, 0.0, out2);
  if (threadIdx.x == 0) {
    partials[3 * blockIdx.x] = t0;
    partials[3 * blockIdx.x + 1] = t1;
    partials[3 * blockIdx.x + 2] = out2[0];
  }
}

// One block: fixed-order reduction of the partials, then the decision (solver.py:1077-1096) and the stop rule.
__global__ void k_mag_decide(const double* __restrict__ partials, int nblocks, mmx_rhs_state* S) {
  double a0 = 0.0, a1 = 0.0, a2 = 0.0;
  for (int i = threadIdx.x; i < nblocks; i += blockDim.x) {
    a0 += partials[3 * i];
    a1 += partials[3 * i + 1];
    a2 += partials[3 * i + 2];
  }
  double out2[2];
  block_reduce_2<double>(a0, a1, out2);
  const double dd2 = out2[0], en2 = out2[1];
  __syncthreads();
  block_reduce_2<double>(a2, 0.0, out2);
  if (threadIdx.x != 0) return;
  const double e2 = out2[0];
  if (!S->active) {
    S->reserved[0] = 0;
    return;
  }
  S->reserved[0] = 1;
  const double nu = sqrt(dd2);
  S->iteration += 1;
  S->last_norm = nu;
  const double prev = S->prev_norm;
  if (prev == 0.0) {  // Python float division by zero in solver.py:1079
    S->status = MMX_STATUS_ZERODIV;
    S->active = 0;
    S->accepted = 0;
    return;
  }
  if (nu / prev < 1.0) {
    S->prev_norm = nu;
    S->field_norm = sqrt(en2);
    S->accepted = 1;
  } else {
    S->alpha_im = 1.5 * S->alpha_im;  // solver.py:1092
    S->rejections += 1;
    S->field_norm = sqrt(e2);
    S->accepted = 0;
  }
  const double fn = S->field_norm;
  S->residue = fn > 0.0 ? S->prev_norm / fn : (S->prev_norm == 0.0 ? 0.0 : INFINITY);
  S->active = ((double)S->iteration < S->maxiter) && (S->residue > S->rtol);
}

// E += d when this iteration ran and its update was accepted
template <class R>
__global__ void k_mag_accept(cpx<R>* __restrict__ E, const cpx<R>* __restrict__ d, const mmx_rhs_state* st,
                             int64_t n) {
  if (!st->reserved[0] || !st->accepted) return;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    E[i] = E[i] + d[i];
}
