// Complex arithmetic on float2 / double2 and the small-radix DFT butterflies of the shared-memory FFT.
//
// The DFT butterflies follow the textbook definitions X_k = sum_n x_n exp(-+2 pi i n k / r) (sign -1 forward,
// +1 inverse, unscaled) written out for r = 2, 3, 4, 5, 8, 16; other radices use the direct O(r^2) sum with roots
// taken from the transform's twiddle table.  The constants are the exact algebraic values of the roots of unity.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

template <class R> struct cpx_s;
template <> struct cpx_s<float> { using type = float2; };
template <> struct cpx_s<double> { using type = double2; };
template <class R> using cpx = typename cpx_s<R>::type;

template <class R> __host__ __device__ __forceinline__ cpx<R> mkc(R re, R im) {
  cpx<R> z;
  z.x = re;
  z.y = im;
  return z;
}

#define MMX_CPX_OPS(V, R)                                                                                   \
  __host__ __device__ __forceinline__ V operator+(V a, V b) { return mkc<R>(a.x + b.x, a.y + b.y); }       \
  __host__ __device__ __forceinline__ V operator-(V a, V b) { return mkc<R>(a.x - b.x, a.y - b.y); }       \
  __host__ __device__ __forceinline__ V operator-(V a) { return mkc<R>(-a.x, -a.y); }                      \
  __host__ __device__ __forceinline__ V operator*(V a, V b) {                                               \
    return mkc<R>(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);                                            \
  }                                                                                                         \
  __host__ __device__ __forceinline__ V operator*(V a, R s) { return mkc<R>(a.x * s, a.y * s); }           \
  __host__ __device__ __forceinline__ V operator*(R s, V a) { return mkc<R>(a.x * s, a.y * s); }           \
  __host__ __device__ __forceinline__ V& operator+=(V& a, V b) {                                            \
    a.x += b.x;                                                                                             \
    a.y += b.y;                                                                                             \
    return a;                                                                                               \
  }                                                                                                         \
  __host__ __device__ __forceinline__ V& operator-=(V& a, V b) {                                            \
    a.x -= b.x;                                                                                             \
    a.y -= b.y;                                                                                             \
    return a;                                                                                               \
  }                                                                                                         \
  __host__ __device__ __forceinline__ V conjc(V a) { return mkc<R>(a.x, -a.y); }                           \
  __host__ __device__ __forceinline__ R norm2c(V a) { return a.x * a.x + a.y * a.y; }                      \
  /* multiply by -i (s = -1) or +i (s = +1) */                                                              \
  __host__ __device__ __forceinline__ V mul_i(V a, int s) { return s < 0 ? mkc<R>(a.y, -a.x) : mkc<R>(-a.y, a.x); }

MMX_CPX_OPS(float2, float)
MMX_CPX_OPS(double2, double)

// complex division a / b
template <class V> __host__ __device__ __forceinline__ V divc(V a, V b) {
  auto d = b.x * b.x + b.y * b.y;
  V r;
  r.x = (a.x * b.x + a.y * b.y) / d;
  r.y = (a.y * b.x - a.x * b.y) / d;
  return r;
}

template <class R, class V> __device__ __forceinline__ V castc(V a) { return a; }
__device__ __forceinline__ float2 to_c32(double2 a) { return make_float2((float)a.x, (float)a.y); }
__device__ __forceinline__ float2 to_c32(float2 a) { return a; }
__device__ __forceinline__ double2 to_c64(float2 a) { return make_double2(a.x, a.y); }
__device__ __forceinline__ double2 to_c64(double2 a) { return a; }
template <class R> __device__ __forceinline__ cpx<R> to_prec(float2 a);
template <class R> __device__ __forceinline__ cpx<R> to_prec(double2 a);
template <> __device__ __forceinline__ float2 to_prec<float>(float2 a) { return a; }
template <> __device__ __forceinline__ float2 to_prec<float>(double2 a) { return to_c32(a); }
template <> __device__ __forceinline__ double2 to_prec<double>(float2 a) { return to_c64(a); }
template <> __device__ __forceinline__ double2 to_prec<double>(double2 a) { return a; }

// ---------------------------------------------------------------------------------------------------------------
// Butterflies.  DIR = -1 forward (exp(-2 pi i nk/r)), +1 inverse.  In place on u[0..r-1].
// ---------------------------------------------------------------------------------------------------------------
#define MMX_SQRT1_2 0.70710678118654752440084436210484903928
#define MMX_SQRT3_2 0.86602540378443864676372317075293618347
#define MMX_C5_1 0.30901699437494742410229341718281905886   // cos(2 pi / 5) = (sqrt 5 - 1) / 4
#define MMX_C5_2 -0.80901699437494742410229341718281905886  // cos(4 pi / 5) = -(sqrt 5 + 1) / 4
#define MMX_S5_1 0.95105651629515357211643933337938214340   // sin(2 pi / 5)
#define MMX_S5_2 0.58778525229247312916870595463907276860   // sin(4 pi / 5)
#define MMX_C16_1 0.92387953251128675612818318939678828682  // cos(pi / 8)
#define MMX_S16_1 0.38268343236508977172845998403039886676  // sin(pi / 8)

template <class R, int DIR> __device__ __forceinline__ void bfly2(cpx<R>* u) {
  cpx<R> a = u[0], b = u[1];
  u[0] = a + b;
  u[1] = a - b;
}

template <class R, int DIR> __device__ __forceinline__ void bfly4v(cpx<R>& a, cpx<R>& b, cpx<R>& c, cpx<R>& d) {
  cpx<R> t0 = a + c, t1 = a - c, t2 = b + d, t3 = mul_i(b - d, DIR);
  a = t0 + t2;
  c = t0 - t2;
  b = t1 + t3;
  d = t1 - t3;
}

template <class R, int DIR> __device__ __forceinline__ void bfly4(cpx<R>* u) { bfly4v<R, DIR>(u[0], u[1], u[2], u[3]); }

template <class R, int DIR> __device__ __forceinline__ void bfly3(cpx<R>* u) {
  cpx<R> a = u[0], b = u[1], c = u[2];
  cpx<R> t = b + c;
  cpx<R> m = a - (R)0.5 * t;
  cpx<R> s = mul_i(b - c, DIR) * (R)MMX_SQRT3_2;
  u[0] = a + t;
  u[1] = m + s;
  u[2] = m - s;
}

template <class R, int DIR> __device__ __forceinline__ void bfly5(cpx<R>* u) {
  cpx<R> a = u[0];
  cpx<R> t1 = u[1] + u[4], t2 = u[2] + u[3], t3 = u[1] - u[4], t4 = u[2] - u[3];
  cpx<R> m1 = a + (R)MMX_C5_1 * t1 + (R)MMX_C5_2 * t2;
  cpx<R> m2 = a + (R)MMX_C5_2 * t1 + (R)MMX_C5_1 * t2;
  cpx<R> s1 = mul_i((R)MMX_S5_1 * t3 + (R)MMX_S5_2 * t4, DIR);
  cpx<R> s2 = mul_i((R)MMX_S5_2 * t3 - (R)MMX_S5_1 * t4, DIR);
  u[0] = a + t1 + t2;
  u[1] = m1 + s1;
  u[4] = m1 - s1;
  u[2] = m2 + s2;
  u[3] = m2 - s2;
}

// multiply by exp(DIR * 2 pi i / 8) (k = 1), exp(DIR * 2 pi i 2/8) = DIR*i (k = 2), exp(DIR * 2 pi i 3/8) (k = 3)
template <class R, int DIR> __device__ __forceinline__ cpx<R> w8_1(cpx<R> a) {
  // (1 + DIR i) / sqrt 2
  return mkc<R>((a.x - DIR * a.y) * (R)MMX_SQRT1_2, (a.y + DIR * a.x) * (R)MMX_SQRT1_2);
}
template <class R, int DIR> __device__ __forceinline__ cpx<R> w8_3(cpx<R> a) {
  // (-1 + DIR i) / sqrt 2
  return mkc<R>((-a.x - DIR * a.y) * (R)MMX_SQRT1_2, (-a.y + DIR * a.x) * (R)MMX_SQRT1_2);
}

template <class R, int DIR> __device__ __forceinline__ void bfly8(cpx<R>* u) {
  // even/odd split: E = DFT4(u0,u2,u4,u6), O = DFT4(u1,u3,u5,u7); X_k = E_k + w^k O_k, X_{k+4} = E_k - w^k O_k
  cpx<R> e0 = u[0], e1 = u[2], e2 = u[4], e3 = u[6];
  cpx<R> o0 = u[1], o1 = u[3], o2 = u[5], o3 = u[7];
  bfly4v<R, DIR>(e0, e1, e2, e3);
  bfly4v<R, DIR>(o0, o1, o2, o3);
  o1 = w8_1<R, DIR>(o1);
  o2 = mul_i(o2, DIR);
  o3 = w8_3<R, DIR>(o3);
  u[0] = e0 + o0;
  u[4] = e0 - o0;
  u[1] = e1 + o1;
  u[5] = e1 - o1;
  u[2] = e2 + o2;
  u[6] = e2 - o2;
  u[3] = e3 + o3;
  u[7] = e3 - o3;
}

template <class R, int DIR> __device__ __forceinline__ void bfly16(cpx<R>* u) {
  // x[n1 + 4 n2]: DFT4 over n2 for each n1, twiddle w16^(n1 k2), DFT4 over n1; X[k2 + 4 k1]
  cpx<R> y[16];
#pragma unroll
  for (int n1 = 0; n1 < 4; ++n1) {
    cpx<R> a = u[n1], b = u[n1 + 4], c = u[n1 + 8], d = u[n1 + 12];
    bfly4v<R, DIR>(a, b, c, d);
    y[n1 * 4 + 0] = a;
    y[n1 * 4 + 1] = b;
    y[n1 * 4 + 2] = c;
    y[n1 * 4 + 3] = d;
  }
  const R c1 = (R)MMX_C16_1, s1 = (R)MMX_S16_1, h = (R)MMX_SQRT1_2;
  // w16^m = cos(2 pi m/16) + DIR i sin(2 pi m/16)
  // n1 = 1: k2 = 1,2,3 -> m = 1,2,3 ; n1 = 2: m = 2,4,6 ; n1 = 3: m = 3,6,9
  auto tw = [&](cpx<R> a, R c, R s) { return mkc<R>(a.x * c - DIR * a.y * s, a.y * c + DIR * a.x * s); };
  y[5] = tw(y[5], c1, s1);
  y[6] = tw(y[6], h, h);
  y[7] = tw(y[7], s1, c1);
  y[9] = tw(y[9], h, h);
  y[10] = mul_i(y[10], DIR);
  y[11] = tw(y[11], -h, h);
  y[13] = tw(y[13], s1, c1);
  y[14] = tw(y[14], -h, h);
  y[15] = tw(y[15], -c1, -s1);
#pragma unroll
  for (int k2 = 0; k2 < 4; ++k2) {
    cpx<R> a = y[0 * 4 + k2], b = y[1 * 4 + k2], c = y[2 * 4 + k2], d = y[3 * 4 + k2];
    bfly4v<R, DIR>(a, b, c, d);
    u[k2 + 0] = a;
    u[k2 + 4] = b;
    u[k2 + 8] = c;
    u[k2 + 12] = d;
  }
}

// Direct DFT of odd prime radix r with roots from the length-n forward table tw (tw[t] = exp(-2 pi i t / n)).
template <class R, int RAD, int DIR> __device__ __forceinline__ void bfly_direct(cpx<R>* u, const cpx<R>* tw, int n) {
  cpx<R> x[RAD];
#pragma unroll
  for (int q = 0; q < RAD; ++q) x[q] = u[q];
  const int step = n / RAD;
#pragma unroll
  for (int k = 0; k < RAD; ++k) {
    cpx<R> acc = x[0];
#pragma unroll
    for (int q = 1; q < RAD; ++q) {
      cpx<R> w = tw[((q * k) % RAD) * step];
      if (DIR > 0) w = conjc(w);
      acc += x[q] * w;
    }
    u[k] = acc;
  }
}

template <class R, int RAD, int DIR> __device__ __forceinline__ void bfly(cpx<R>* u, const cpx<R>* tw, int n) {
  if constexpr (RAD == 2) bfly2<R, DIR>(u);
  else if constexpr (RAD == 3) bfly3<R, DIR>(u);
  else if constexpr (RAD == 4) bfly4<R, DIR>(u);
  else if constexpr (RAD == 5) bfly5<R, DIR>(u);
  else if constexpr (RAD == 8) bfly8<R, DIR>(u);
  else if constexpr (RAD == 16) bfly16<R, DIR>(u);
  else bfly_direct<R, RAD, DIR>(u, tw, n);
}
