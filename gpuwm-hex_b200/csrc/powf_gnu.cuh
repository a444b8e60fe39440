// glibc-order single-precision powf for positive normal bases, on the device.
//
// MPAS computes the Exner function with the host libm powf; the reference
// reproduces GNU libc 2.39's order (hexcore/native_powf.py:18,128), which is
// the published algorithm of Arm optimized-routines v21.02 math/powf.c
// (MIT licence, Copyright (c) 2017-2019 Arm Limited): log2(x) from a 16-entry
// table of (1/c, log2 c) and a degree-5 polynomial, y*log2(x), then exp2 from a
// 32-entry table of 2^(i/32) and a cubic, in double precision without fused
// multiply-adds (this file is compiled with -fmad=false in strict builds and
// uses explicit __dadd_rn/__dmul_rn so that no build contracts it), then
// rounded to binary32.  The log table and polynomials are Arm's published
// constants; the exp2 table is 2^(i/32) with i<<47 subtracted from its bits.
#pragma once
#include <stdint.h>

namespace hexdyn_powf {

static __device__ __constant__ double kLog2Tab[16][2] = {
    {0x1.661ec79f8f3bep+0, -0x1.efec65b963019p-2},
    {0x1.571ed4aaf883dp+0, -0x1.b0b6832d4fca4p-2},
    {0x1.49539f0f010bp+0, -0x1.7418b0a1fb77bp-2},
    {0x1.3c995b0b80385p+0, -0x1.39de91a6dcf7bp-2},
    {0x1.30d190c8864a5p+0, -0x1.01d9bf3f2b631p-2},
    {0x1.25e227b0b8eap+0, -0x1.97c1d1b3b7afp-3},
    {0x1.1bb4a4a1a343fp+0, -0x1.2f9e393af3c9fp-3},
    {0x1.12358f08ae5bap+0, -0x1.960cbbf788d5cp-4},
    {0x1.0953f419900a7p+0, -0x1.a6f9db6475fcep-5},
    {0x1p+0, 0x0p+0},
    {0x1.e608cfd9a47acp-1, 0x1.338ca9f24f53dp-4},
    {0x1.ca4b31f026aap-1, 0x1.476a9543891bap-3},
    {0x1.b2036576afce6p-1, 0x1.e840b4ac4e4d2p-3},
    {0x1.9c2d163a1aa2dp-1, 0x1.40645f0c6651cp-2},
    {0x1.886e6037841edp-1, 0x1.88e9c2c1b9ff8p-2},
    {0x1.767dcf5534862p-1, 0x1.ce0a44eb17bccp-2},
};

static __device__ __constant__ double kLog2Poly[5] = {
    0x1.27616c9496e0bp-2, -0x1.71969a075c67ap-2, 0x1.ec70a6ca7baddp-2,
    -0x1.7154748bef6c8p-1, 0x1.71547652ab82bp0,
};

// bits(2^(i/32) rounded to double) - (i << 47); generated from that
// definition with 60-digit decimal arithmetic (a CPU test re-derives it).
#define HEXDYN_EXP2_TABLE                                                                      \
  0x3ff0000000000000ull, 0x3fefd9b0d3158574ull, 0x3fefb5586cf9890full, 0x3fef9301d0125b51ull, \
  0x3fef72b83c7d517bull, 0x3fef54873168b9aaull, 0x3fef387a6e756238ull, 0x3fef1e9df51fdee1ull, \
  0x3fef06fe0a31b715ull, 0x3feef1a7373aa9cbull, 0x3feedea64c123422ull, 0x3feece086061892dull, \
  0x3feebfdad5362a27ull, 0x3feeb42b569d4f82ull, 0x3feeab07dd485429ull, 0x3feea47eb03a5585ull, \
  0x3feea09e667f3bcdull, 0x3fee9f75e8ec5f74ull, 0x3feea11473eb0187ull, 0x3feea589994cce13ull, \
  0x3feeace5422aa0dbull, 0x3feeb737b0cdc5e5ull, 0x3feec49182a3f090ull, 0x3feed503b23e255dull, \
  0x3feee89f995ad3adull, 0x3feeff76f2fb5e47ull, 0x3fef199bdd85529cull, 0x3fef3720dcef9069ull, \
  0x3fef5818dcfba487ull, 0x3fef7c97337b9b5full, 0x3fefa4afa2a490daull, 0x3fefd0765b6e4540ull
static __device__ __constant__ uint64_t kExp2Tab[32] = {HEXDYN_EXP2_TABLE};

// Returns powf(x, y) for positive normal x; *bad is set for any other base.
__device__ __forceinline__ float powf_gnu(float x, float y, int* bad) {
  uint32_t ix = __float_as_uint(x);
  if (!(ix >= 0x00800000u && ix < 0x7f800000u)) {
    *bad = 1;
    return __int_as_float(0x7fc00000);
  }
  uint32_t tmp = ix - 0x3f330000u;
  int i = (int)((tmp >> 19) % 16u);
  uint32_t top = tmp & 0xff800000u;
  double z = (double)__uint_as_float(ix - top);
  double k = (double)(((int32_t)top) >> 23);
  double invc = kLog2Tab[i][0], logc = kLog2Tab[i][1];
  double r = __dadd_rn(__dmul_rn(z, invc), -1.0);
  double y0 = __dadd_rn(logc, k);
  double r2 = __dmul_rn(r, r);
  double r4 = __dmul_rn(r2, r2);
  double yl = __dadd_rn(__dmul_rn(kLog2Poly[0], r), kLog2Poly[1]);
  double p = __dadd_rn(__dmul_rn(kLog2Poly[2], r), kLog2Poly[3]);
  double q = __dadd_rn(__dmul_rn(kLog2Poly[4], r), y0);
  q = __dadd_rn(__dmul_rn(p, r2), q);
  yl = __dadd_rn(__dmul_rn(yl, r4), q);
  double xd = __dmul_rn((double)y, yl);
  if (fabs(xd) > 1000.0) {
    *bad = 1;
    return __int_as_float(0x7fc00000);
  }
  const double shift = 0x1.8p+47;
  double kd = __dadd_rn(xd, shift);
  uint64_t ki = (uint64_t)__double_as_longlong(kd);
  double rr = __dadd_rn(xd, -__dadd_rn(kd, -shift));
  uint64_t t = kExp2Tab[ki % 32u] + (ki << 47);
  double scale = __longlong_as_double((long long)t);
  double zz = __dadd_rn(__dmul_rn(0x1.c6af84b912394p-5, rr), 0x1.ebfce50fac4f3p-3);
  double rr2 = __dmul_rn(rr, rr);
  double yy = __dadd_rn(__dmul_rn(0x1.62e42ff0c52d6p-1, rr), 1.0);
  yy = __dadd_rn(__dmul_rn(zz, rr2), yy);
  return __double2float_rn(__dmul_rn(yy, scale));
}

}  // namespace hexdyn_powf
