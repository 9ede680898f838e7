// dft.cuh -- in-register complex DFTs with compile-time twiddles (sm_100a).
//
// Building blocks of the spectrometer FFT.  Every small DFT works on an
// array of float2 held in registers, natural order in and out, forward sign
// (W_R = exp(-2 pi i / R)), unscaled -- the convention of the reference's
// forward real DFT (ippsDFTFwd_RToPerm_32f with IPP_FFT_DIV_INV_BY_N,
// src/IA-32/TaskCoreIPP.cpp:116,430).  Composite sizes run a Stockham
// autosort over register passes; all indices and twiddles are compile-time
// constants, so trivial rotations (1, -i, -1, i, 45-degree) cost no multiply.
#pragma once

#include <cuda_runtime.h>
#include <type_traits>

namespace sws {

// ---------------------------------------------------------------------------
// compile-time trigonometry (Taylor series on an exactly reduced argument)
// ---------------------------------------------------------------------------
__host__ __device__ constexpr double cx_sin_small(double x)
{
   double x2 = x * x, term = x, sum = x;
   for (int n = 1; n < 14; n++) {
      term *= -x2 / ((2.0 * n) * (2.0 * n + 1.0));
      sum += term;
   }
   return sum;
}
__host__ __device__ constexpr double cx_cos_small(double x)
{
   double x2 = x * x, term = 1.0, sum = 1.0;
   for (int n = 1; n < 14; n++) {
      term *= -x2 / ((2.0 * n - 1.0) * (2.0 * n));
      sum += term;
   }
   return sum;
}
// cos(2 pi m / R), with the quadrant chosen from the integers m, R
__host__ __device__ constexpr double cx_cos2pi(long m, long R)
{
   m %= R;
   if (m < 0) m += R;
   const double PI = 3.14159265358979323846264338327950288;
   long k = ((8 * m) / R + 1) / 2 % 4;
   double r = 2.0 * PI * (double)m / (double)R - (double)k * (PI / 2);
   double c = cx_cos_small(r), s = cx_sin_small(r);
   return k == 0 ? c : k == 1 ? -s : k == 2 ? -c : s;
}
// sin(2 pi m / R) = cos(2 pi (4m - R) / (4R))
__host__ __device__ constexpr double cx_sin2pi(long m, long R) { return cx_cos2pi(4 * m - R, 4 * R); }

template <int I, int N, typename F>
__device__ __forceinline__ void static_for(F &&f)
{
   if constexpr (I < N) {
      f(std::integral_constant<int, I>{});
      static_for<I + 1, N>(f);
   }
}

// ---------------------------------------------------------------------------
// complex helpers
// ---------------------------------------------------------------------------
__device__ __forceinline__ float2 cadd(float2 a, float2 b) { return make_float2(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ float2 csub(float2 a, float2 b) { return make_float2(a.x - b.x, a.y - b.y); }
// The same sums as one packed two-lane instruction (add/sub.rn.f32x2, sm_100);
// for operands that are plain register pairs, where no swizzle is needed.
__device__ __forceinline__ float2 padd(float2 a, float2 b)
{
   float2 d;
   asm("{\n .reg .b64 ra, rb, rd;\n mov.b64 ra, {%2, %3};\n mov.b64 rb, {%4, %5};\n"
       " add.rn.f32x2 rd, ra, rb;\n mov.b64 {%0, %1}, rd;\n}\n"
       : "=f"(d.x), "=f"(d.y) : "f"(a.x), "f"(a.y), "f"(b.x), "f"(b.y));
   return d;
}
__device__ __forceinline__ float2 psub(float2 a, float2 b)
{
   float2 d;
   asm("{\n .reg .b64 ra, rb, rd;\n mov.b64 ra, {%2, %3};\n mov.b64 rb, {%4, %5};\n"
       " sub.rn.f32x2 rd, ra, rb;\n mov.b64 {%0, %1}, rd;\n}\n"
       : "=f"(d.x), "=f"(d.y) : "f"(a.x), "f"(a.y), "f"(b.x), "f"(b.y));
   return d;
}
__device__ __forceinline__ float2 cmul(float2 a, float2 w)
{
   return make_float2(fmaf(a.x, w.x, -a.y * w.y), fmaf(a.x, w.y, a.y * w.x));
}
__device__ __forceinline__ float2 cmulconj(float2 a, float2 w)  // a * conj(w)
{
   return make_float2(fmaf(a.x, w.x, a.y * w.y), fmaf(a.y, w.x, -a.x * w.y));
}
__device__ __forceinline__ float2 mul_negi(float2 a) { return make_float2(a.y, -a.x); }  // a * (-i)
__device__ __forceinline__ float2 mul_posi(float2 a) { return make_float2(-a.y, a.x); }  // a * (+i)

// a * W_R^m with compile-time m, R
template <int M_, int R>
__device__ __forceinline__ float2 twmul(float2 a)
{
   constexpr int m = ((M_ % R) + R) % R;
   if constexpr (m == 0) {
      return a;
   } else if constexpr (4 * m == R) {
      return mul_negi(a);
   } else if constexpr (2 * m == R) {
      return make_float2(-a.x, -a.y);
   } else if constexpr (4 * m == 3 * R) {
      return mul_posi(a);
   } else if constexpr (8 * m == R) {
      constexpr float c = 0.70710678118654752440f;
      return make_float2((a.x + a.y) * c, (a.y - a.x) * c);
   } else if constexpr (8 * m == 3 * R) {
      constexpr float c = 0.70710678118654752440f;
      return make_float2((a.y - a.x) * c, -(a.x + a.y) * c);
   } else if constexpr (8 * m == 5 * R) {
      constexpr float c = 0.70710678118654752440f;
      return make_float2(-(a.x + a.y) * c, (a.x - a.y) * c);
   } else if constexpr (8 * m == 7 * R) {
      constexpr float c = 0.70710678118654752440f;
      return make_float2((a.x - a.y) * c, (a.x + a.y) * c);
   } else {
      constexpr float wr = (float)cx_cos2pi(m, R);
      constexpr float wi = -(float)cx_sin2pi(m, R);
      return cmul(a, make_float2(wr, wi));
   }
}

// ---------------------------------------------------------------------------
// small DFTs
// ---------------------------------------------------------------------------
template <int R>
struct DFT;

template <>
struct DFT<1> {
   __device__ __forceinline__ static void run(float2 *) {}
};

template <>
struct DFT<2> {
   __device__ __forceinline__ static void run(float2 *v)
   {
      float2 a = v[0], b = v[1];
      v[0] = padd(a, b);
      v[1] = psub(a, b);
   }
};

template <>
struct DFT<3> {
   __device__ __forceinline__ static void run(float2 *v)
   {
      constexpr float s = 0.86602540378443864676f;  // sin(2 pi / 3)
      float2 t1 = padd(v[1], v[2]), t2 = psub(v[1], v[2]);
      float2 m = make_float2(fmaf(-0.5f, t1.x, v[0].x), fmaf(-0.5f, t1.y, v[0].y));
      v[0] = padd(v[0], t1);
      v[1] = make_float2(fmaf(s, t2.y, m.x), fmaf(-s, t2.x, m.y));
      v[2] = make_float2(fmaf(-s, t2.y, m.x), fmaf(s, t2.x, m.y));
   }
};

template <>
struct DFT<4> {
   __device__ __forceinline__ static void run(float2 *v)
   {
      float2 s0 = padd(v[0], v[2]), s1 = psub(v[0], v[2]);
      float2 s2 = padd(v[1], v[3]), s3 = psub(v[1], v[3]);
      v[0] = padd(s0, s2);
      v[2] = psub(s0, s2);
      v[1] = cadd(s1, mul_negi(s3));
      v[3] = csub(s1, mul_negi(s3));
   }
};

template <>
struct DFT<5> {
   __device__ __forceinline__ static void run(float2 *v)
   {
      constexpr float c1 = 0.30901699437494742410f;   // cos(2 pi / 5)
      constexpr float c2 = -0.80901699437494742410f;  // cos(4 pi / 5)
      constexpr float s1 = 0.95105651629515357212f;   // sin(2 pi / 5)
      constexpr float s2 = 0.58778525229247312917f;   // sin(4 pi / 5)
      float2 t1 = padd(v[1], v[4]), t2 = padd(v[2], v[3]);
      float2 t3 = psub(v[1], v[4]), t4 = psub(v[2], v[3]);
      float2 x0 = v[0];
      float2 a1 = make_float2(fmaf(c2, t2.x, fmaf(c1, t1.x, x0.x)), fmaf(c2, t2.y, fmaf(c1, t1.y, x0.y)));
      float2 a2 = make_float2(fmaf(c1, t2.x, fmaf(c2, t1.x, x0.x)), fmaf(c1, t2.y, fmaf(c2, t1.y, x0.y)));
      float2 b1 = make_float2(fmaf(s1, t3.x, s2 * t4.x), fmaf(s1, t3.y, s2 * t4.y));
      float2 b2 = make_float2(fmaf(s2, t3.x, -s1 * t4.x), fmaf(s2, t3.y, -s1 * t4.y));
      v[0] = padd(x0, padd(t1, t2));
      v[1] = cadd(a1, mul_negi(b1));
      v[4] = csub(a1, mul_negi(b1));
      v[2] = cadd(a2, mul_negi(b2));
      v[3] = csub(a2, mul_negi(b2));
   }
};

// smallest prime-ish factor used for register passes (prefers 4)
template <int R>
__host__ __device__ constexpr int first_radix()
{
   if constexpr (R % 4 == 0 && R != 8) return 4;
   else if constexpr (R % 2 == 0) return 2;
   else if constexpr (R % 3 == 0) return 3;
   else if constexpr (R % 5 == 0) return 5;
   else return R;
}

// One Stockham pass of radix r with span Ns over R registers.
template <int R, int Ns, int r>
__device__ __forceinline__ void reg_pass(float2 *v)
{
   float2 t[R];
   constexpr int nb = R / r;
   static_for<0, nb>([&](auto J) {
      constexpr int j = decltype(J)::value;
      constexpr int k = j % Ns;
      float2 u[r];
      static_for<0, r>([&](auto I) {
         constexpr int i = decltype(I)::value;
         u[i] = twmul<k * i * (R / (Ns * r)), R>(v[j + i * nb]);
      });
      DFT<r>::run(u);
      constexpr int d = (j / Ns) * Ns * r + k;
      static_for<0, r>([&](auto I) {
         constexpr int i = decltype(I)::value;
         t[d + i * Ns] = u[i];
      });
   });
#pragma unroll
   for (int i = 0; i < R; i++) v[i] = t[i];
}

template <int R, int Ns>
__device__ __forceinline__ void reg_passes(float2 *v)
{
   if constexpr (Ns < R) {
      constexpr int r = first_radix<R / Ns>();
      reg_pass<R, Ns, r>(v);
      reg_passes<R, Ns * r>(v);
   }
}

template <int R>
struct DFT {
   __device__ __forceinline__ static void run(float2 *v) { reg_passes<R, 1>(v); }
};

}  // namespace sws
