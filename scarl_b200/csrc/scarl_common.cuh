// scarl_common.cuh -- device-side helpers shared by every scarl_b200 kernel:
// complex arithmetic on float2/double2, the Philox4x32-10 counter RNG, the
// Park-Miller jump-ahead, and the exact radix-32 unit-root constants.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

namespace scarl {

template <typename T> struct cplx_of;
template <> struct cplx_of<float> { using type = float2; };
template <> struct cplx_of<double> { using type = double2; };
template <typename T> using cplx_t = typename cplx_of<T>::type;

__device__ __forceinline__ float2 mk(float x, float y) { return make_float2(x, y); }
__device__ __forceinline__ double2 mk(double x, double y) { return make_double2(x, y); }

template <typename C> __device__ __forceinline__ C cadd(C a, C b) { return mk(a.x + b.x, a.y + b.y); }
template <typename C> __device__ __forceinline__ C csub(C a, C b) { return mk(a.x - b.x, a.y - b.y); }
template <typename C> __device__ __forceinline__ C cmul(C a, C b) {
  return mk(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
// a * (+i)
template <typename C> __device__ __forceinline__ C cmul_i(C a) { return mk(-a.y, a.x); }
template <typename C> __device__ __forceinline__ C cconj(C a) { return mk(a.x, -a.y); }
template <typename C, typename T> __device__ __forceinline__ C cscale(C a, T s) { return mk(a.x * s, a.y * s); }

// cos / sin of 2*pi*m/32 for m < 16 (exact to double rounding).
__device__ constexpr double kCos32[16] = {
    1.0, 0.98078528040323044913, 0.92387953251128675613, 0.83146961230254523708,
    0.70710678118654752440, 0.55557023301960222474, 0.38268343236508977173, 0.19509032201612826785,
    0.0, -0.19509032201612826785, -0.38268343236508977173, -0.55557023301960222474,
    -0.70710678118654752440, -0.83146961230254523708, -0.92387953251128675613, -0.98078528040323044913};
__device__ constexpr double kSin32[16] = {
    0.0, 0.19509032201612826785, 0.38268343236508977173, 0.55557023301960222474,
    0.70710678118654752440, 0.83146961230254523708, 0.92387953251128675613, 0.98078528040323044913,
    1.0, 0.98078528040323044913, 0.92387953251128675613, 0.83146961230254523708,
    0.70710678118654752440, 0.55557023301960222474, 0.38268343236508977173, 0.19509032201612826785};

// ---------------------------------------------------------------------------
// Philox4x32-10 (Salmon et al., SC11): counter-based, stateless.
// ---------------------------------------------------------------------------
struct u32x4 { uint32_t x, y, z, w; };

__device__ __forceinline__ u32x4 philox4x32_10(u32x4 c, uint32_t k0, uint32_t k1) {
#pragma unroll
  for (int r = 0; r < 10; ++r) {
    const uint32_t lo0 = 0xD2511F53u * c.x;
    const uint32_t hi0 = __umulhi(0xD2511F53u, c.x);
    const uint32_t lo1 = 0xCD9E8D57u * c.z;
    const uint32_t hi1 = __umulhi(0xCD9E8D57u, c.z);
    u32x4 n;
    n.x = hi1 ^ c.y ^ k0;
    n.y = lo1;
    n.z = hi0 ^ c.w ^ k1;
    n.w = lo0;
    c = n;
    k0 += 0x9E3779B9u;
    k1 += 0xBB67AE85u;
  }
  return c;
}

// The same with the round keys precomputed (ks[r] = k0 + r 0x9E3779B9,
// ks[10 + r] = k1 + r 0xBB67AE85): kernels read them from their parameter
// block instead of rebuilding the schedule per draw.
__device__ __forceinline__ u32x4 philox4x32_10_ks(u32x4 c, const uint32_t* ks) {
#pragma unroll
  for (int r = 0; r < 10; ++r) {
    // each 32 x 32 -> 64-bit product as one wide multiply (both halves)
    const uint64_t p0 = (uint64_t)0xD2511F53u * c.x;
    const uint64_t p1 = (uint64_t)0xCD9E8D57u * c.z;
    u32x4 n;
    n.x = (uint32_t)(p1 >> 32) ^ c.y ^ ks[r];
    n.y = (uint32_t)p1;
    n.z = (uint32_t)(p0 >> 32) ^ c.w ^ ks[10 + r];
    n.w = (uint32_t)p0;
    c = n;
  }
  return c;
}

// Uniform in (0,1) from two 32-bit words: 52 random bits plus a half offset,
// exactly representable, never 0 or 1.
__device__ __forceinline__ double u01_d(uint32_t hi, uint32_t lo) {
  const uint64_t a = ((uint64_t)hi << 32) | lo;
  return (double)(a >> 12) * 0x1p-52 + 0x1p-53;
}
// Canonical standard normals of the padded spectrum.  Modes (kx, ky, kz) and
// (kx, ky, kz + P2/2), kz < P2/2, share one Philox draw
//   Philox(ctr = {c_lo, c_hi, stream, 0}, key),  c = kx + Hx (ky + P1 kz),
// words (x, y) feeding the first and (z, w) the second mode; each word pair
// (a, b) gives u1 = (a + 1/2) 2^-32, u2 = (b + 1/2) 2^-32 and the Box-Muller
// pair r (cos 2 pi u2, sin 2 pi u2), r = sqrt(-2 ln u1).
template <typename T> struct Normals;
template <> struct Normals<double> {
  static __device__ __forceinline__ double2 from(uint32_t a, uint32_t b) {
    const double u1 = (double)a * 0x1p-32 + 0x1p-33;
    const double u2 = (double)b * 0x1p-32 + 0x1p-33;
    const double r = sqrt(-2.0 * log(u1));
    double s, c;
    sincospi(2.0 * u2, &s, &c);
    return make_double2(r * c, r * s);
  }
};
template <> struct Normals<float> {
  // Single precision, hardware transcendentals: u1 is formed with one
  // rounding (relative error 2^-24, so small u1 keep their digits); the
  // phase is reduced to (-pi, pi) where __sincosf is accurate, and the
  // half-turn folded back by the sign.
  static __device__ __forceinline__ float2 from(uint32_t a, uint32_t b) {
    const float u1 = __fmaf_rn((float)a, 0x1p-32f, 0x1p-33f);
    const float u2 = __fmaf_rn((float)b, 0x1p-32f, 0x1p-33f);
    const float r = sqrtf(-2.0f * __logf(u1));
    float s, c;
    __sincosf(6.28318530717958647692f * (u2 - 0.5f), &s, &c);
    return make_float2(-r * c, -r * s);
  }
};

// ---------------------------------------------------------------------------
// Park-Miller (16807, 2^31-1): state after n steps from s, s in [0, 2^31-1).
// pw[b] = 16807^(2^b) mod (2^31-1).
// ---------------------------------------------------------------------------
__device__ __forceinline__ uint32_t pm_mulmod(uint32_t a, uint32_t b) {
  const uint64_t p = (uint64_t)a * b;
  uint64_t r = (p & 0x7FFFFFFFull) + (p >> 31);
  r = (r & 0x7FFFFFFFull) + (r >> 31);
  return (r == 0x7FFFFFFFull) ? 0u : (uint32_t)r;
}
__device__ __forceinline__ uint32_t pm_jump(uint32_t s, uint64_t n, const uint32_t* __restrict__ pw) {
  uint32_t r = s;
  int b = 0;
  while (n) {
    if (n & 1) r = pm_mulmod(r, pw[b]);
    n >>= 1;
    ++b;
  }
  return r;
}

}  // namespace scarl
