// Mode synthesis and detection of the scattering matrix on the device: the plane-wave modes of a transverse plane
// are the propagating entries of its spectrum, so
//   synthesis (srcvec2freespace, matrix.py:528-610): spectrum[row][mode index m] = coefficient[row][m], then a
//       forward transform over the transverse axes (mmx_fftn);
//   detection (detfield2detvec, matrix.py:685-755): an inverse transform over the transverse axes, then
//       coefficient[row][m] = spectrum[row][mode index m].
// A row is one (right-hand side, component, plane) transverse plane of `row_len` samples; `idx` lists the spectrum
// position of every mode.  The kernels below do the scatter and the gather as grid-stride loops over all
// (row, mode) pairs.
#pragma once
#include "mmx_complex.cuh"

// out[r][idx[m]] = (conj ? conj(in[r][m]) : in[r][m]); the other entries of `out` are left as they are
template <class R>
__global__ void k_mode_scatter(const cpx<R>* __restrict__ in, const int64_t* __restrict__ idx, int64_t nmodes,
                               int64_t nrows, int64_t row_len, int conj, cpx<R>* __restrict__ out) {
  const int64_t total = nrows * nmodes;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < total; i += (int64_t)gridDim.x * blockDim.x) {
    const int64_t r = i / nmodes, m = i - r * nmodes;
    const int64_t k = idx[m];
    if (k < 0 || k >= row_len) continue;  // an index outside the row is skipped (the host validates the table)
    cpx<R> v = in[i];
    if (conj) v = conjc(v);
    out[r * row_len + k] = v;
  }
}

// out[r][m] = (conj ? conj(in[r][idx[m]]) : in[r][idx[m]])
template <class R>
__global__ void k_mode_gather(const cpx<R>* __restrict__ in, const int64_t* __restrict__ idx, int64_t nmodes,
                              int64_t nrows, int64_t row_len, int conj, cpx<R>* __restrict__ out) {
  const int64_t total = nrows * nmodes;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < total; i += (int64_t)gridDim.x * blockDim.x) {
    const int64_t r = i / nmodes, m = i - r * nmodes;
    const int64_t k = idx[m];
    cpx<R> v = (k >= 0 && k < row_len) ? in[r * row_len + k] : mkc<R>(0, 0);
    if (conj) v = conjc(v);
    out[i] = v;
  }
}
