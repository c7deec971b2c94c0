// Complex arithmetic and register-resident small DFTs for the H|psi> kernels.
//
// Sign convention: S = +1 is the backward transform (e^{+i G.r}, what the
// reference calls MODE = -1 in Src/fft/_cfft/cfft_wf_c16.f), S = -1 is the
// forward transform (e^{-i G.r}, MODE = +1).
//
// DFT<R,S,T>::run(v) transforms R values held in registers, in place, output
// in natural order. R in {1,2,3,4,5,6,8,9,10,12,16}: radix 2/3/4/5 butterflies
// and compile-time two-level compositions of them. The composite twiddles are
// compile-time constants evaluated with a Taylor series after exact octant
// reduction of the rational angle k/R (our own routine, error < 1 ulp).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

namespace cpwb {

template <typename T> struct C2;
template <> struct alignas(16) C2<double> { double x, y; };
template <> struct alignas(8) C2<float> { float x, y; };

template <typename T> __host__ __device__ __forceinline__ C2<T> mk(T a, T b) { C2<T> r; r.x = a; r.y = b; return r; }
template <typename T> __device__ __forceinline__ C2<T> operator+(C2<T> a, C2<T> b) { return mk<T>(a.x + b.x, a.y + b.y); }
template <typename T> __device__ __forceinline__ C2<T> operator-(C2<T> a, C2<T> b) { return mk<T>(a.x - b.x, a.y - b.y); }
template <typename T> __device__ __forceinline__ C2<T> cmul(C2<T> a, C2<T> b) {
  return mk<T>(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
// a * conj(b)
template <typename T> __device__ __forceinline__ C2<T> cmulc(C2<T> a, C2<T> b) {
  return mk<T>(a.x * b.x + a.y * b.y, a.y * b.x - a.x * b.y);
}
template <typename T> __device__ __forceinline__ C2<T> scal(C2<T> a, T s) { return mk<T>(a.x * s, a.y * s); }
// A real constant for products in T. In FP32 the constant is carried as hi + lo and applied
// with one FMA, so that its rounding leaves no systematic gain: a constant rounded once to
// FP32 (sqrt(3)/2, sqrt(1/2), cos(2 pi/5), ...) scales every value it touches by the same
// relative error (up to ~3e-8), a bias the forward/inverse pair of transforms accumulates.
template <typename T> struct K;
template <> struct K<double> {
  double v;
  __host__ __device__ constexpr K(double c) : v(c) {}
  __device__ __forceinline__ double mul(double x) const { return x * v; }
};
template <> struct K<float> {
  float h, l;
  __host__ __device__ constexpr K(double c) : h((float)c), l((float)(c - (double)(float)c)) {}
  __device__ __forceinline__ float mul(float x) const { return fmaf(x, h, x * l); }
};
template <typename T> __device__ __forceinline__ C2<T> kscal(C2<T> a, K<T> k) { return mk<T>(k.mul(a.x), k.mul(a.y)); }

// FP32 complex add, subtract and split-constant scaling as packed two-lane instructions
// (add/sub/mul/fma .rn.f32x2, sm_100): the same per-component IEEE rounding as the scalar
// forms above, half the instructions in the butterflies of the issue-bound FP32 transforms.
__device__ __forceinline__ unsigned long long f32x2_bits(C2<float> a) {
  unsigned long long r;
  asm("mov.b64 %0, {%1, %2};" : "=l"(r) : "f"(a.x), "f"(a.y));
  return r;
}
__device__ __forceinline__ C2<float> f32x2_val(unsigned long long r) {
  C2<float> a;
  asm("mov.b64 {%0, %1}, %2;" : "=f"(a.x), "=f"(a.y) : "l"(r));
  return a;
}
__device__ __forceinline__ C2<float> operator+(C2<float> a, C2<float> b) {
  unsigned long long d;
  asm("add.rn.f32x2 %0, %1, %2;" : "=l"(d) : "l"(f32x2_bits(a)), "l"(f32x2_bits(b)));
  return f32x2_val(d);
}
__device__ __forceinline__ C2<float> operator-(C2<float> a, C2<float> b) {
  unsigned long long d;
  asm("sub.rn.f32x2 %0, %1, %2;" : "=l"(d) : "l"(f32x2_bits(a)), "l"(f32x2_bits(b)));
  return f32x2_val(d);
}
template <> __device__ __forceinline__ C2<float> kscal<float>(C2<float> a, K<float> k) {
  unsigned long long t, d;
  const unsigned long long x = f32x2_bits(a);
  asm("mul.rn.f32x2 %0, %1, %2;" : "=l"(t) : "l"(x), "l"(f32x2_bits(mk<float>(k.l, k.l))));
  asm("fma.rn.f32x2 %0, %1, %2, %3;" : "=l"(d) : "l"(x), "l"(f32x2_bits(mk<float>(k.h, k.h))), "l"(t));
  return f32x2_val(d);
}
// a * (c + i s) with split constants
__device__ __forceinline__ C2<double> kcmul(C2<double> a, K<double> c, K<double> s) {
  return mk<double>(a.x * c.v - a.y * s.v, a.x * s.v + a.y * c.v);
}
__device__ __forceinline__ C2<float> kcmul(C2<float> a, K<float> c, K<float> s) {
  const float re_lo = a.x * c.l - a.y * s.l, im_lo = a.x * s.l + a.y * c.l;
  return mk<float>(fmaf(a.x, c.h, fmaf(-a.y, s.h, re_lo)), fmaf(a.x, s.h, fmaf(a.y, c.h, im_lo)));
}

// multiply by i*S (S = +1 or -1)
template <int S, typename T> __device__ __forceinline__ C2<T> mul_iS(C2<T> a) {
  return S > 0 ? mk<T>(-a.y, a.x) : mk<T>(a.y, -a.x);
}

// ---------------- compile-time trigonometry ----------------
namespace ct {
constexpr double PI = 3.14159265358979323846264338327950288;
constexpr double taylor_sin(double x) {
  double term = x, sum = x;
  for (int n = 1; n < 14; ++n) { term *= -x * x / ((2 * n) * (2 * n + 1)); sum += term; }
  return sum;
}
constexpr double taylor_cos(double x) {
  double term = 1.0, sum = 1.0;
  for (int n = 1; n < 14; ++n) { term *= -x * x / ((2 * n - 1) * (2 * n)); sum += term; }
  return sum;
}
// cos and sin of 2*pi*k/R, reduced to [0, pi/4] with exact rational folds.
struct CS { double c, s; };
constexpr CS cos_sin_frac(long k, long R) {
  k %= R; if (k < 0) k += R;
  // f = k/R in [0,1). Work with numerator over 8R to keep folds exact.
  long num = 8 * k, den = 8 * R;           // f = num/den
  double sgn_s = 1.0, sgn_c = 1.0;
  if (2 * num > den) { num = den - num; sgn_s = -1.0; }          // f -> 1-f : sin flips
  bool swap = false;
  if (4 * num > den) { num = den / 2 - num; sgn_c = -sgn_c; }    // f -> 1/2-f : cos flips
  if (8 * num > den) { num = den / 4 - num; swap = true; }       // f -> 1/4-f : swap sin/cos
  double x = 2.0 * PI * (double)num / (double)den;
  double c = taylor_cos(x), s = taylor_sin(x);
  if (swap) { double t = c; c = s; s = t; }
  return CS{sgn_c * c, sgn_s * s};
}
template <int R> struct Tw {
  double c[R], s[R];
  constexpr Tw() : c(), s() {
    for (int k = 0; k < R; ++k) { CS v = cos_sin_frac(k, R); c[k] = v.c; s[k] = v.s; }
  }
};
}  // namespace ct

// ---------------- register DFTs ----------------
template <int R, int S, typename T> struct DFT;

template <int S, typename T> struct DFT<1, S, T> { static __device__ __forceinline__ void run(C2<T>*) {} };

template <int S, typename T> struct DFT<2, S, T> {
  static __device__ __forceinline__ void run(C2<T>* v) {
    C2<T> a = v[0] + v[1], b = v[0] - v[1];
    v[0] = a; v[1] = b;
  }
};

template <int S, typename T> struct DFT<3, S, T> {
  static __device__ __forceinline__ void run(C2<T>* v) {
    constexpr K<T> h(0.866025403784438646763723170752936183);  // sqrt(3)/2
    C2<T> t1 = v[1] + v[2];
    C2<T> t2 = v[0] - scal<T>(t1, T(0.5));
    C2<T> t3 = mul_iS<S, T>(kscal<T>(v[1] - v[2], h));
    v[0] = v[0] + t1;
    v[1] = t2 + t3;
    v[2] = t2 - t3;
  }
};

template <int S, typename T> struct DFT<4, S, T> {
  static __device__ __forceinline__ void run(C2<T>* v) {
    C2<T> a0 = v[0] + v[2], a1 = v[0] - v[2];
    C2<T> b0 = v[1] + v[3], b1 = mul_iS<S, T>(v[1] - v[3]);
    v[0] = a0 + b0; v[2] = a0 - b0; v[1] = a1 + b1; v[3] = a1 - b1;
  }
};

template <int S, typename T> struct DFT<5, S, T> {
  static __device__ __forceinline__ void run(C2<T>* v) {
    constexpr K<T> c1(0.309016994374947424102293417182819059);   // cos(2pi/5)
    constexpr K<T> c2(-0.809016994374947424102293417182819059);  // cos(4pi/5)
    constexpr K<T> s1(0.951056516295153572116439333379382143);   // sin(2pi/5)
    constexpr K<T> s2(0.587785252292473129168705954639072769);   // sin(4pi/5)
    C2<T> t1 = v[1] + v[4], t2 = v[2] + v[3], t3 = v[1] - v[4], t4 = v[2] - v[3];
    C2<T> a1 = v[0] + kscal<T>(t1, c1) + kscal<T>(t2, c2);
    C2<T> a2 = v[0] + kscal<T>(t1, c2) + kscal<T>(t2, c1);
    C2<T> b1 = mul_iS<S, T>(kscal<T>(t3, s1) + kscal<T>(t4, s2));
    C2<T> b2 = mul_iS<S, T>(kscal<T>(t3, s2) - kscal<T>(t4, s1));
    v[0] = v[0] + t1 + t2;
    v[1] = a1 + b1; v[4] = a1 - b1;
    v[2] = a2 + b2; v[3] = a2 - b2;
  }
};

// Two-level composition R = A*B in registers: input index B*n1+n2, output k1+A*k2.
template <int A, int B, int S, typename T> struct DFTComp {
  static __device__ __forceinline__ void run(C2<T>* v) {
    constexpr int R = A * B;
    constexpr ct::Tw<R> tw{};
    C2<T> t[R];
#pragma unroll
    for (int n2 = 0; n2 < B; ++n2) {
      C2<T> u[A];
#pragma unroll
      for (int n1 = 0; n1 < A; ++n1) u[n1] = v[B * n1 + n2];
      DFT<A, S, T>::run(u);
#pragma unroll
      for (int k1 = 0; k1 < A; ++k1) {
        const int m = (n2 * k1) % R;
        if (m == 0) {
          t[k1 * B + n2] = u[k1];
        } else if (4 * m == R) {                 // W = i*S
          t[k1 * B + n2] = mul_iS<S, T>(u[k1]);
        } else if (2 * m == R) {                 // W = -1
          t[k1 * B + n2] = mk<T>(-u[k1].x, -u[k1].y);
        } else if (4 * m == 3 * R) {             // W = -i*S
          t[k1 * B + n2] = mul_iS<-S, T>(u[k1]);
        } else {
          t[k1 * B + n2] = kcmul(u[k1], K<T>(tw.c[m]), K<T>(S * tw.s[m]));
        }
      }
    }
#pragma unroll
    for (int k1 = 0; k1 < A; ++k1) {
      C2<T> u[B];
#pragma unroll
      for (int n2 = 0; n2 < B; ++n2) u[n2] = t[k1 * B + n2];
      DFT<B, S, T>::run(u);
#pragma unroll
      for (int k2 = 0; k2 < B; ++k2) v[k1 + A * k2] = u[k2];
    }
  }
};

template <int S, typename T> struct DFT<6, S, T> : DFTComp<2, 3, S, T> {};
template <int S, typename T> struct DFT<8, S, T> : DFTComp<2, 4, S, T> {};
template <int S, typename T> struct DFT<9, S, T> : DFTComp<3, 3, S, T> {};
template <int S, typename T> struct DFT<10, S, T> : DFTComp<2, 5, S, T> {};
template <int S, typename T> struct DFT<12, S, T> : DFTComp<3, 4, S, T> {};
template <int S, typename T> struct DFT<16, S, T> : DFTComp<4, 4, S, T> {};

// Radices the runtime dispatch accepts (a line length n is split n = r1*r2).
__host__ __device__ constexpr bool radix_ok(int r) {
  return r == 1 || r == 2 || r == 3 || r == 4 || r == 5 || r == 6 || r == 8 || r == 9 ||
         r == 10 || r == 12 || r == 16;
}

// Radix dispatch: with RC > 0 the radix is the compile-time RC, otherwise the
// warp-uniform runtime r selects the instantiation: f(IC<R>{}).
template <int N> struct IC { static constexpr int value = N; };
template <typename F> __device__ __forceinline__ void radix_dispatch(int r, F&& f) {
  switch (r) {
    case 1: f(IC<1>{}); break;
    case 2: f(IC<2>{}); break;
    case 3: f(IC<3>{}); break;
    case 4: f(IC<4>{}); break;
    case 5: f(IC<5>{}); break;
    case 6: f(IC<6>{}); break;
    case 8: f(IC<8>{}); break;
    case 9: f(IC<9>{}); break;
    case 10: f(IC<10>{}); break;
    case 12: f(IC<12>{}); break;
    case 16: f(IC<16>{}); break;
    default: break;
  }
}
template <int RC, typename F> __device__ __forceinline__ void with_radix(int r, F&& f) {
  if constexpr (RC > 0) {
    f(IC<RC>{});
  } else {
    radix_dispatch(r, static_cast<F&&>(f));
  }
}

}  // namespace cpwb
