// pmcmc_rng.cuh -- counter-based tape generator (device side).
//
// The reference draws its MALA tape (xi_t ~ N(0, I_D), u_t ~ U(0,1)) and the
// Hutchinson probes from one Julia MersenneTwister on the host
// (interface.jl:334-358, DEER.jl:298-325, 407, 412).  That stream cannot be
// reproduced, and it makes block k+1's tape depend on how many Newton
// iterations block k took.  Here the tape is a pure function of
// (seed, block, t, d) -- Philox4x32-10 (Salmon et al., SC'11) -- so every
// column is generated where it is consumed, inside the sweep kernels, and the
// host oracle regenerates exactly the same bits.
//
// Normals: Box-Muller on two 23-bit uniforms.  log and sin/cos are this
// project's own FP32 polynomials (atanh series for log, Taylor series for
// sin/cos on [-pi/4, pi/4]) written with explicitly rounded intrinsics, so the
// device result is bit-identical to the host C implementation compiled with
// -ffp-contract=off.
//
// Counter layout (key = seed):
//   xi  : ctr = {d/4, t, block, 1}          -> 4 normals for d = 4j..4j+3
//   u   : ctr = {0,   t, block, 2}          -> word 0
//   z   : ctr = {d/128, t, block, 3 | probe<<4 | iter<<12} -> bit d%128
#pragma once
#include <cstdint>

namespace pmcmc {

constexpr uint32_t kPhiloxM0 = 0xD2511F53u;
constexpr uint32_t kPhiloxM1 = 0xCD9E8D57u;
constexpr uint32_t kPhiloxW0 = 0x9E3779B9u;
constexpr uint32_t kPhiloxW1 = 0xBB67AE85u;
constexpr uint32_t kTagXi = 1u, kTagU = 2u, kTagZ = 3u;

struct U4 {
  uint32_t x, y, z, w;
};

__device__ __forceinline__ U4 philox4x32_10(uint32_t c0, uint32_t c1, uint32_t c2, uint32_t c3,
                                            uint32_t k0, uint32_t k1) {
#pragma unroll
  for (int r = 0; r < 10; ++r) {
    if (r > 0) {
      k0 += kPhiloxW0;
      k1 += kPhiloxW1;
    }
    const uint32_t lo0 = kPhiloxM0 * c0, hi0 = __umulhi(kPhiloxM0, c0);
    const uint32_t lo1 = kPhiloxM1 * c2, hi1 = __umulhi(kPhiloxM1, c2);
    const uint32_t n0 = hi1 ^ c1 ^ k0, n2 = hi0 ^ c3 ^ k1;
    c0 = n0;
    c1 = lo1;
    c2 = n2;
    c3 = lo0;
  }
  return U4{c0, c1, c2, c3};
}

// (2k+1) * 2^-24 with k = bits >> 9: exact in FP32, strictly inside (0, 1).
__device__ __forceinline__ float tape_u01(uint32_t bits) {
  return __fmul_rn(static_cast<float>(2u * (bits >> 9) + 1u), 0x1p-24f);
}

// ln(x) for x in [2^-24, 1].
__device__ __forceinline__ float tape_log(float x) {
  const uint32_t b = __float_as_uint(x);
  int e = static_cast<int>((b >> 23) & 0xffu) - 127;
  float m = __uint_as_float((b & 0x7fffffu) | 0x3f800000u);
  if (m > 0x1.6a09e6p+0f) {
    m = __fmul_rn(m, 0.5f);
    e += 1;
  }
  const float num = __fsub_rn(m, 1.0f);
  const float den = __fadd_rn(m, 1.0f);
  const float s = __fdiv_rn(num, den);
  const float s2 = __fmul_rn(s, s);
  float p = 0x1.745d18p-4f;
  p = __fmaf_rn(p, s2, 0x1.c71c72p-4f);
  p = __fmaf_rn(p, s2, 0x1.24924ap-3f);
  p = __fmaf_rn(p, s2, 0x1.99999ap-3f);
  p = __fmaf_rn(p, s2, 0x1.555556p-2f);
  const float t = __fmul_rn(2.0f, s);
  const float ts2 = __fmul_rn(t, s2);
  const float lnm = __fmaf_rn(ts2, p, t);
  return __fmaf_rn(static_cast<float>(e), 0x1.62e430p-1f, lnm);
}

// sin(2 pi u), cos(2 pi u) for u in (0, 1).
__device__ __forceinline__ void tape_sincos2pi(float u, float& s_out, float& c_out) {
  const float q4 = __fmul_rn(u, 4.0f);
  const float k = rintf(q4);
  const float f = __fsub_rn(q4, k);
  const float phi = __fmul_rn(f, 0x1.921fb6p+0f);
  const float p2 = __fmul_rn(phi, phi);
  float sp = 0x1.71de3ap-19f;
  sp = __fmaf_rn(sp, p2, -0x1.a01a02p-13f);
  sp = __fmaf_rn(sp, p2, 0x1.111112p-7f);
  sp = __fmaf_rn(sp, p2, -0x1.555556p-3f);
  const float pp = __fmul_rn(phi, p2);
  const float sn = __fmaf_rn(pp, sp, phi);
  float cp = -0x1.27e4fcp-22f;
  cp = __fmaf_rn(cp, p2, 0x1.a01a02p-16f);
  cp = __fmaf_rn(cp, p2, -0x1.6c16c2p-10f);
  cp = __fmaf_rn(cp, p2, 0x1.555556p-5f);
  cp = __fmaf_rn(cp, p2, -0.5f);
  const float cs = __fmaf_rn(p2, cp, 1.0f);
  switch (static_cast<int>(k) & 3) {
    case 0: s_out = sn; c_out = cs; break;
    case 1: s_out = cs; c_out = -sn; break;
    case 2: s_out = -sn; c_out = -cs; break;
    default: s_out = -cs; c_out = sn; break;
  }
}

__device__ __forceinline__ void box_muller(uint32_t b1, uint32_t b2, float& n0, float& n1) {
  const float u1 = tape_u01(b1), u2 = tape_u01(b2);
  const float L = tape_log(u1);
  const float r = __fsqrt_rn(__fmul_rn(-2.0f, L));
  float s, c;
  tape_sincos2pi(u2, s, c);
  n0 = __fmul_rn(r, c);
  n1 = __fmul_rn(r, s);
}

struct TapeKey {
  uint32_t k0, k1, block;
  __host__ __device__ TapeKey(uint64_t seed, uint64_t blk)
      : k0(static_cast<uint32_t>(seed)), k1(static_cast<uint32_t>(seed >> 32)),
        block(static_cast<uint32_t>(blk)) {}
};

// Four tape normals for d = 4j .. 4j+3 of column t.
__device__ __forceinline__ void tape_xi4(const TapeKey& key, uint32_t j, uint32_t t, float n[4]) {
  const U4 o = philox4x32_10(j, t, key.block, kTagXi, key.k0, key.k1);
  box_muller(o.x, o.y, n[0], n[1]);
  box_muller(o.z, o.w, n[2], n[3]);
}

__device__ __forceinline__ float tape_u(const TapeKey& key, uint32_t t) {
  const U4 o = philox4x32_10(0u, t, key.block, kTagU, key.k0, key.k1);
  return tape_u01(o.x);
}

// 128 Rademacher bits for d in [128 j, 128 j + 128) of column t.
__device__ __forceinline__ U4 probe_bits(const TapeKey& key, uint32_t j, uint32_t t, int probe,
                                         int iter) {
  const uint32_t tag = kTagZ | (static_cast<uint32_t>(probe) << 4) |
                       (static_cast<uint32_t>(iter) << 12);
  return philox4x32_10(j, t, key.block, tag, key.k0, key.k1);
}

__device__ __forceinline__ uint32_t u4_word(const U4& o, int w) {
  return w == 0 ? o.x : (w == 1 ? o.y : (w == 2 ? o.z : o.w));
}

}  // namespace pmcmc
