// Building blocks of the iteration for magnetic and bi-(an)isotropic media (reference solver.py:531-552).
//
// The magnetic susceptibility operator is chi(x) = chi_EE x + chi_HE D x + D(chi_EH x + chi_HH D x), with D the
// spectral curl i k x (backend/__init__.py:472-509; k of the k0-scaled grid).  It is applied twice per iteration,
// so an iteration costs four curls (FFT pairs) plus the Green function's FFT pair; the host composes it from the
// batched FFT (mmx_fftn) and the pointwise kernels below:
//   k_curl_ft:   F -> i k x F for a 3-component spectrum [3][N]
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

template <class R>
__global__ void k_curl_ft(const cpx<R>* __restrict__ F, cpx<R>* __restrict__ out, KGrid g, const R* kv0,
                          const R* kv1, const R* kv2) {
  const R* kv[3] = {kv0, kv1, kv2};
  const int64_t N = g.N;
  for (int64_t v = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; v < N; v += (int64_t)gridDim.x * blockDim.x) {
    R k[3];
    k_of_voxel<R>(g, kv, v, k);
    const cpx<R> f0 = F[v], f1 = F[N + v], f2 = F[2 * N + v];
    // (k x F)_d = k_{d+1} F_{d-1} - k_{d-1} F_{d+1}; axes beyond the grid have k = 0
    const cpx<R> c0 = k[1] * f2 - k[2] * f1;
    const cpx<R> c1 = k[2] * f0 - k[0] * f2;
    const cpx<R> c2 = k[0] * f1 - k[1] * f0;
    out[v] = mul_i(c0, 1);
    out[N + v] = mul_i(c1, 1);
    out[2 * N + v] = mul_i(c2, 1);
  }
}

template <class R>
__global__ void k_green_ft(cpx<R>* __restrict__ F, KGrid g, const R* kv0, const R* kv1, const R* kv2, R ar, R ai) {
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

// coef: [ee_a, ee_b, eh_f, he_f, hh_f] as complex pairs: chi_EE(alpha) = ee_a chi_EE0 + ee_b I, the others scaled
template <class R>
__global__ void k_chi_mix(const cpx<R>* __restrict__ x, const cpx<R>* __restrict__ d, const cpx<R>* __restrict__ ee,
                          const cpx<R>* __restrict__ eh, const cpx<R>* __restrict__ he, const cpx<R>* __restrict__ hh,
                          cpx<R> ee_a, cpx<R> ee_b, cpx<R> eh_f, cpx<R> he_f, cpx<R> hh_f, cpx<R>* __restrict__ u,
                          cpx<R>* __restrict__ w, int64_t N) {
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
