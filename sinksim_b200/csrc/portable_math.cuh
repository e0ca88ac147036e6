// Portable transcendental functions: sin, cos and pow computed by the published algorithms of fdlibm 5.3 (Sun
// Microsystems, freely distributable: s_sin.c, s_cos.c, k_sin.c, k_cos.c, the small and medium argument paths of
// e_rem_pio2.c, e_pow.c, s_scalbn.c), restated here as host-and-device functions. Every step is an IEEE-754
// double operation that rounds once (the translation units are compiled without contraction: -fmad=false for
// nvcc, -ffp-contract=off for the host compiler), so the CPU and the GPU produce the same bits as the C fdlibm.
//
// These are the "portable" math of the reference engine (engine/include/sinksim/kernel/math.hpp:41-46): sin and
// cos in the pose (kernel/frame.hpp:10-21), pow in the Villemonte weir law (kernel/flows.hpp:59). The parity tests
// hold them bit for bit against the reference's vendored fdlibm over the sample sets of
// tests/test_portable_math.cpp of the reference (SplitMix64, seed 20261008).
#pragma once

#include <cstdint>

#if defined(__CUDACC__)
#define SSB_HD __host__ __device__ __forceinline__
#else
#define SSB_HD inline
#endif

#if !defined(__CUDA_ARCH__)
#include <cmath>
#include <cstring>
#endif

namespace ssb::pm {

// ----------------------------------------------------------------------------- IEEE words of a double

SSB_HD std::int32_t high_word(double x) {
#if defined(__CUDA_ARCH__)
  return __double2hiint(x);
#else
  std::uint64_t b;
  std::memcpy(&b, &x, 8);
  return static_cast<std::int32_t>(static_cast<std::uint32_t>(b >> 32));
#endif
}

SSB_HD std::uint32_t low_word(double x) {
#if defined(__CUDA_ARCH__)
  return static_cast<std::uint32_t>(__double2loint(x));
#else
  std::uint64_t b;
  std::memcpy(&b, &x, 8);
  return static_cast<std::uint32_t>(b);
#endif
}

SSB_HD double from_words(std::int32_t hi, std::uint32_t lo) {
#if defined(__CUDA_ARCH__)
  return __hiloint2double(hi, static_cast<int>(lo));
#else
  const std::uint64_t b = (static_cast<std::uint64_t>(static_cast<std::uint32_t>(hi)) << 32) | lo;
  double x;
  std::memcpy(&x, &b, 8);
  return x;
#endif
}

// x with its low word cleared: the "head" of a two-piece number, exact in products with 24-bit factors.
SSB_HD double clear_low(double x) { return from_words(high_word(x), 0u); }

SSB_HD double abs_of(double x) { return from_words(high_word(x) & 0x7fffffff, low_word(x)); }

SSB_HD double sqrt_rn(double x) {
#if defined(__CUDA_ARCH__)
  return __dsqrt_rn(x);
#else
  return std::sqrt(x);
#endif
}

// ----------------------------------------------------------------------------- scalbn (s_scalbn.c)

SSB_HD double copy_sign(double x, double y) {
  return from_words(static_cast<std::int32_t>((static_cast<std::uint32_t>(high_word(x)) & 0x7fffffffu) |
                                              (static_cast<std::uint32_t>(high_word(y)) & 0x80000000u)),
                    low_word(x));
}

// x * 2^n by exponent arithmetic, with fdlibm's overflow, underflow and subnormal handling.
SSB_HD double scale2(double x, int n) {
  const double two54 = 1.80143985094819840000e+16, twom54 = 5.55111512312578270212e-17;
  const double big = 1.0e+300, small = 1.0e-300;
  std::int32_t hx = high_word(x);
  std::int32_t e = (hx & 0x7ff00000) >> 20;
  if (e == 0) {                                     // zero or subnormal
    if (((hx & 0x7fffffff) | static_cast<std::int32_t>(low_word(x))) == 0) return x;
    x *= two54;
    hx = high_word(x);
    e = ((hx & 0x7ff00000) >> 20) - 54;
    if (n < -50000) return small * x;
  }
  if (e == 0x7ff) return x + x;                     // inf or NaN
  e += n;
  if (e > 0x7fe) return big * copy_sign(big, x);    // overflow
  const std::int32_t keep = hx & static_cast<std::int32_t>(0x800fffff);
  if (e > 0) return from_words(keep | static_cast<std::int32_t>(static_cast<std::uint32_t>(e) << 20), low_word(x));
  if (e <= -54) {
    if (n > 50000) return big * copy_sign(big, x);
    return small * copy_sign(small, x);             // underflow
  }
  e += 54;                                          // subnormal result
  return from_words(keep | static_cast<std::int32_t>(static_cast<std::uint32_t>(e) << 20), low_word(x)) * twom54;
}

// ----------------------------------------------------------------------------- kernels on [-pi/4, pi/4] (k_sin.c, k_cos.c)

// sin(x + y) for |x| <= pi/4, y the tail of x; tail_used = 0 when y is known to be zero.
SSB_HD double sin_kernel(double x, double y, int tail_used) {
  const double S1 = -1.66666666666666324348e-01, S2 = 8.33333333332248946124e-03, S3 = -1.98412698298579493134e-04,
               S4 = 2.75573137070700676789e-06, S5 = -2.50507602534068634195e-08, S6 = 1.58969099521155010221e-10;
  const std::int32_t ix = high_word(x) & 0x7fffffff;
  if (ix < 0x3e400000 && static_cast<int>(x) == 0) return x;   // |x| < 2^-27: sin x = x (inexact)
  const double z = x * x;
  const double v = z * x;
  const double r = S2 + z * (S3 + z * (S4 + z * (S5 + z * S6)));
  if (tail_used == 0) return x + v * (S1 + z * r);
  return x - ((z * (0.5 * y - v * r) - y) - v * S1);
}

// cos(x + y) for |x| <= pi/4.
SSB_HD double cos_kernel(double x, double y) {
  const double C1 = 4.16666666666666019037e-02, C2 = -1.38888888888741095749e-03, C3 = 2.48015872894767294178e-05,
               C4 = -2.75573143513906633035e-07, C5 = 2.08757232129817482790e-09, C6 = -1.13596475577881948265e-11;
  const std::int32_t ix = high_word(x) & 0x7fffffff;
  if (ix < 0x3e400000 && static_cast<int>(x) == 0) return 1.0;  // |x| < 2^-27
  const double z = x * x;
  const double r = z * (C1 + z * (C2 + z * (C3 + z * (C4 + z * (C5 + z * C6)))));
  if (ix < 0x3FD33333) return 1.0 - (0.5 * z - (z * r - x * y));  // |x| < 0.3
  // cos(x) = (1 - q) - ((z/2 - q) - (z r - x y)), with q = |x|/4 rounded to its high word, or 0.28125 above 0.78125
  const double q = ix > 0x3fe90000 ? 0.28125 : from_words(ix - 0x00200000, 0u);
  return (1.0 - q) - ((0.5 * z - q) - (z * r - x * y));
}

// ----------------------------------------------------------------------------- argument reduction (e_rem_pio2.c)

// Reduces x by a multiple n of pi/2 with |x| <= 2^19 pi/2, returning n and the remainder as y0 + y1. Larger
// arguments need the Payne-Hanek path of fdlibm (k_rem_pio2.c), which this engine never reaches: its angles are
// clamped at 1.4 rad. *ok is cleared for them.
SSB_HD int reduce_half_pi(double x, double& y0, double& y1, bool& ok) {
  const double invpio2 = 6.36619772367581382433e-01;
  const double pio2_1 = 1.57079632673412561417e+00, pio2_1t = 6.07710050650619224932e-11;
  const double pio2_2 = 6.07710050630396597660e-11, pio2_2t = 2.02226624879595063154e-21;
  const double pio2_3 = 2.02226624871116645580e-21, pio2_3t = 8.47842766036889956997e-32;
  const std::int32_t hx = high_word(x), ix = hx & 0x7fffffff;
  ok = true;
  if (ix <= 0x3fe921fb) { y0 = x; y1 = 0; return 0; }
  if (ix < 0x4002d97c) {                            // |x| < 3pi/4: one subtraction of pi/2
    const double sgn = hx > 0 ? 1.0 : -1.0;
    const double ax = hx > 0 ? x : -x;
    double z = ax - pio2_1;
    if (ix != 0x3ff921fb) {                         // 33+53 bits of pi/2 are enough
      y0 = z - pio2_1t;
      y1 = (z - y0) - pio2_1t;
    } else {                                        // near pi/2: 33+33+53 bits
      z -= pio2_2;
      y0 = z - pio2_2t;
      y1 = (z - y0) - pio2_2t;
    }
    if (hx < 0) { y0 = -y0; y1 = -y1; }
    return static_cast<int>(sgn);
  }
  if (ix > 0x413921fb) { ok = false; y0 = x; y1 = 0; return 0; }
  // medium arguments: n = nearest integer to |x| 2/pi, then up to three pieces of pi/2
  const double t = abs_of(x);
  const int n = static_cast<int>(t * invpio2 + 0.5);
  const double fn = static_cast<double>(n);
  double r = t - fn * pio2_1;
  double w = fn * pio2_1t;
  // high words of the first 32 multiples of pi/2: an argument that shares one may cancel in r - w
  bool cancel;
  {
    const std::int32_t nh[32] = {0x3FF921FB, 0x400921FB, 0x4012D97C, 0x401921FB, 0x401F6A7A, 0x4022D97C, 0x4025FDBB, 0x402921FB,
                                 0x402C463A, 0x402F6A7A, 0x4031475C, 0x4032D97C, 0x40346B9C, 0x4035FDBB, 0x40378FDB, 0x403921FB,
                                 0x403AB41B, 0x403C463A, 0x403DD85A, 0x403F6A7A, 0x40407E4C, 0x4041475C, 0x4042106C, 0x4042D97C,
                                 0x4043A28C, 0x40446B9C, 0x404534AC, 0x4045FDBB, 0x4046C6CB, 0x40478FDB, 0x404858EB, 0x404921FB};
    cancel = !(n < 32 && ix != nh[n - 1]);
  }
  y0 = r - w;
  if (cancel) {
    const std::int32_t ex = ix >> 20;
    std::int32_t gap = ex - ((high_word(y0) >> 20) & 0x7ff);
    if (gap > 16) {                                 // second iteration with 33+33 bits of pi/2
      double u = r;
      w = fn * pio2_2;
      r = u - w;
      w = fn * pio2_2t - ((u - r) - w);
      y0 = r - w;
      gap = ex - ((high_word(y0) >> 20) & 0x7ff);
      if (gap > 49) {                               // third iteration, 151 bits of pi/2
        u = r;
        w = fn * pio2_3;
        r = u - w;
        w = fn * pio2_3t - ((u - r) - w);
        y0 = r - w;
      }
    }
  }
  y1 = (r - y0) - w;
  if (hx < 0) { y0 = -y0; y1 = -y1; return -n; }
  return n;
}

SSB_HD double sin(double x) {
  const std::int32_t ix = high_word(x) & 0x7fffffff;
  if (ix <= 0x3fe921fb) return sin_kernel(x, 0.0, 0);
  if (ix >= 0x7ff00000) return x - x;               // inf or NaN
  double y0, y1;
  bool ok;
  const int n = reduce_half_pi(x, y0, y1, ok);
  if (!ok) {
#if defined(__CUDA_ARCH__)
    return ::sin(x);
#else
    return std::sin(x);
#endif
  }
  switch (n & 3) {
    case 0: return sin_kernel(y0, y1, 1);
    case 1: return cos_kernel(y0, y1);
    case 2: return -sin_kernel(y0, y1, 1);
    default: return -cos_kernel(y0, y1);
  }
}

SSB_HD double cos(double x) {
  const std::int32_t ix = high_word(x) & 0x7fffffff;
  if (ix <= 0x3fe921fb) return cos_kernel(x, 0.0);
  if (ix >= 0x7ff00000) return x - x;
  double y0, y1;
  bool ok;
  const int n = reduce_half_pi(x, y0, y1, ok);
  if (!ok) {
#if defined(__CUDA_ARCH__)
    return ::cos(x);
#else
    return std::cos(x);
#endif
  }
  switch (n & 3) {
    case 0: return cos_kernel(y0, y1);
    case 1: return -sin_kernel(y0, y1, 1);
    case 2: return -cos_kernel(y0, y1);
    default: return sin_kernel(y0, y1, 1);
  }
}

// ----------------------------------------------------------------------------- pow (e_pow.c)

// log2(ax) as t1 + t2, t1 with a cleared low word, for |y| <= 2^31 (the general path of e_pow.c step 1).
SSB_HD void log2_two_piece(double ax, std::int32_t ix, double& t1, double& t2) {
  const double two53 = 9007199254740992.0;
  const double L1 = 5.99999999999994648725e-01, L2 = 4.28571428578550184252e-01, L3 = 3.33333329818377432918e-01,
               L4 = 2.72728123808534006489e-01, L5 = 2.30660745775561754067e-01, L6 = 2.06975017800338417784e-01;
  const double cp = 9.61796693925975554329e-01, cp_h = 9.61796700954437255859e-01, cp_l = -7.02846165095275826516e-09;
  const double dp_h1 = 5.84962487220764160156e-01, dp_l1 = 1.35003920212974897128e-08;
  std::int32_t n = 0;
  if (ix < 0x00100000) {                            // subnormal x: normalise
    ax *= two53;
    n -= 53;
    ix = high_word(ax);
  }
  n += (ix >> 20) - 0x3ff;
  const std::int32_t j = ix & 0x000fffff;
  ix = j | 0x3ff00000;                              // mantissa in [1, 2)
  int k;
  if (j <= 0x3988E) k = 0;                          // m < sqrt(3/2): expand about 1
  else if (j < 0xBB67A) k = 1;                      // m < sqrt(3): expand about 1.5
  else { k = 0; n += 1; ix -= 0x00100000; }         // m >= sqrt(3): halve it
  ax = from_words(ix, low_word(ax));
  const double bp = k ? 1.5 : 1.0;
  const double dph = k ? dp_h1 : 0.0, dpl = k ? dp_l1 : 0.0;
  // s = (m - bp) / (m + bp) in two pieces
  double u = ax - bp;
  double v = 1.0 / (ax + bp);
  const double s = u * v;
  const double s_h = clear_low(s);
  double t_h = from_words(((ix >> 1) | 0x20000000) + 0x00080000 + static_cast<std::int32_t>(static_cast<std::uint32_t>(k) << 18), 0u);
  double t_l = ax - (t_h - bp);
  const double s_l = v * ((u - s_h * t_h) - s_h * t_l);
  // log(m) = 2 s + 2/3 s^3 + s^4 R(s^2), the series scaled by 3/2
  double s2 = s * s;
  double r = s2 * s2 * (L1 + s2 * (L2 + s2 * (L3 + s2 * (L4 + s2 * (L5 + s2 * L6)))));
  r += s_l * (s_h + s);
  s2 = s_h * s_h;
  t_h = clear_low(3.0 + s2 + r);
  t_l = r - ((t_h - 3.0) - s2);
  u = s_h * t_h;
  v = s_l * t_h + t_l * s;
  const double p_h = clear_low(u + v);
  const double p_l = v - (p_h - u);
  // times 2/(3 ln 2), plus the exponent and the log2 of bp
  const double z_h = cp_h * p_h;
  const double z_l = cp_l * p_h + p_l * cp + dpl;
  const double t = static_cast<double>(n);
  t1 = clear_low(((z_h + z_l) + dph) + t);
  t2 = z_l - (((t1 - t) - dph) - z_h);
}

SSB_HD double pow(double x, double y) {
  const double huge = 1.0e300, tiny = 1.0e-300;
  const double P1 = 1.66666666666666019037e-01, P2 = -2.77777777770155933842e-03, P3 = 6.61375632143793436117e-05,
               P4 = -1.65339022054652515390e-06, P5 = 4.13813679705723846039e-08;
  const double lg2 = 6.93147180559945286227e-01, lg2_h = 6.93147182464599609375e-01, lg2_l = -1.90465429995776804525e-09;
  const double ovt = 8.0085662595372944372e-0017;
  const double ivln2 = 1.44269504088896338700e+00, ivln2_h = 1.44269502162933349609e+00, ivln2_l = 1.92596299112661746887e-08;

  const std::int32_t hx = high_word(x), hy = high_word(y);
  const std::uint32_t lx = low_word(x), ly = low_word(y);
  const std::int32_t ix = hx & 0x7fffffff, iy = hy & 0x7fffffff;

  if ((static_cast<std::uint32_t>(iy) | ly) == 0) return 1.0;                              // x^0
  if (ix > 0x7ff00000 || (ix == 0x7ff00000 && lx != 0) || iy > 0x7ff00000 || (iy == 0x7ff00000 && ly != 0))
    return x + y;                                                                           // NaN operand

  // for negative x: is y an odd integer (1), an even integer (2) or not an integer (0)?
  int yint = 0;
  if (hx < 0) {
    if (iy >= 0x43400000) {
      yint = 2;                                                                             // |y| >= 2^53
    } else if (iy >= 0x3ff00000) {
      const int e = (iy >> 20) - 0x3ff;
      if (e > 20) {
        const std::uint32_t m = ly >> (52 - e);
        if ((m << (52 - e)) == ly) yint = 2 - static_cast<int>(m & 1u);
      } else if (ly == 0) {
        const std::int32_t m = iy >> (20 - e);
        if ((m << (20 - e)) == iy) yint = 2 - (m & 1);
      }
    }
  }

  if (ly == 0) {                                                                            // special y
    if (iy == 0x7ff00000) {                                                                 // y = +-inf
      if (((static_cast<std::uint32_t>(ix - 0x3ff00000)) | lx) == 0) return y - y;         // (+-1)^inf is NaN
      if (ix >= 0x3ff00000) return (hy >= 0) ? y : 0.0;
      return (hy < 0) ? -y : 0.0;
    }
    if (iy == 0x3ff00000) return (hy < 0) ? 1.0 / x : x;                                   // y = +-1
    if (hy == 0x40000000) return x * x;                                                     // y = 2
    if (hy == 0x3fe00000 && hx >= 0) return sqrt_rn(x);                                     // y = 0.5
  }

  double ax = abs_of(x);
  if (lx == 0 && (ix == 0x7ff00000 || ix == 0 || ix == 0x3ff00000)) {                       // x = +-0, +-inf, +-1
    double z = ax;
    if (hy < 0) z = 1.0 / z;
    if (hx < 0) {
      if (((ix - 0x3ff00000) | yint) == 0) z = (z - z) / (z - z);                           // (-1)^non-integer
      else if (yint == 1) z = -z;
    }
    return z;
  }

  const std::int32_t nsign = (hx >> 31) + 1;
  if ((nsign | yint) == 0) return (x - x) / (x - x);                                       // (x<0)^non-integer
  const double sgn = ((nsign | (yint - 1)) == 0) ? -1.0 : 1.0;                              // (x<0)^odd

  double t1, t2;
  if (iy > 0x41e00000) {                                                                    // |y| > 2^31
    if (iy > 0x43f00000) {                                                                  // |y| > 2^64
      if (ix <= 0x3fefffff) return (hy < 0) ? huge * huge : tiny * tiny;
      if (ix >= 0x3ff00000) return (hy > 0) ? huge * huge : tiny * tiny;
    }
    if (ix < 0x3fefffff) return (hy < 0) ? sgn * huge * huge : sgn * tiny * tiny;
    if (ix > 0x3ff00000) return (hy > 0) ? sgn * huge * huge : sgn * tiny * tiny;
    // |1 - x| <= 2^-20: log2(x) from its series about 1
    const double t = ax - 1.0;
    const double w = (t * t) * (0.5 - t * (0.3333333333333333333333 - t * 0.25));
    const double u = ivln2_h * t;
    const double v = t * ivln2_l - w * ivln2;
    t1 = clear_low(u + v);
    t2 = v - (t1 - u);
  } else {
    log2_two_piece(ax, ix, t1, t2);
  }

  // y log2(x) = p_h + p_l, with y split into a 24-bit head and its tail
  const double y1 = clear_low(y);
  double p_l = (y - y1) * t1 + y * t2;
  double p_h = y1 * t1;
  double z = p_l + p_h;
  std::int32_t j = high_word(z);
  std::int32_t i = static_cast<std::int32_t>(low_word(z));
  if (j >= 0x40900000) {                                                                    // z >= 1024
    if (((j - 0x40900000) | i) != 0) return sgn * huge * huge;
    if (p_l + ovt > z - p_h) return sgn * huge * huge;
  } else if ((j & 0x7fffffff) >= 0x4090cc00) {                                              // z <= -1075
    if (((static_cast<std::uint32_t>(j) - 0xc090cc00u) | static_cast<std::uint32_t>(i)) != 0) return sgn * tiny * tiny;
    if (p_l <= z - p_h) return sgn * tiny * tiny;
  }

  // 2^z = 2^n 2^(z - n), n the nearest integer once |z| > 1/2
  i = j & 0x7fffffff;
  int e = (i >> 20) - 0x3ff;
  std::int32_t n = 0;
  if (i > 0x3fe00000) {
    n = j + (0x00100000 >> (e + 1));
    e = ((n & 0x7fffffff) >> 20) - 0x3ff;
    const double tn = from_words(n & ~(0x000fffff >> e), 0u);
    n = ((n & 0x000fffff) | 0x00100000) >> (20 - e);
    if (j < 0) n = -n;
    p_h -= tn;
  }
  double t = clear_low(p_l + p_h);
  const double u = t * lg2_h;
  const double v = (p_l - (t - p_h)) * lg2 + t * lg2_l;
  z = u + v;
  const double w = v - (z - u);
  t = z * z;
  const double c = z - t * (P1 + t * (P2 + t * (P3 + t * (P4 + t * P5))));
  const double r = (z * c) / (c - 2.0) - (w + z * w);
  z = 1.0 - (r - z);
  j = high_word(z) + static_cast<std::int32_t>(static_cast<std::uint32_t>(n) << 20);
  if ((j >> 20) <= 0) z = scale2(z, n);                                                     // subnormal result
  else z = from_words(high_word(z) + static_cast<std::int32_t>(static_cast<std::uint32_t>(n) << 20), low_word(z));
  return sgn * z;
}

}  // namespace ssb::pm
