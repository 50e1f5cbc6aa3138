// Device arithmetic shared by the photon kernels: the counter-based RNG, the Fresnel reflectance
// of an interface and the Henyey-Greenstein spin. Everything here is FP32 except the
// near-critical-angle Fresnel branch, which is FP64.
#pragma once

#include <cstdint>

namespace xmc {

// Philox4x32-10 (Salmon, Moraes, Dror, Shaw: "Parallel random numbers: as easy as 1, 2, 3", SC'11):
// ten rounds of the published round function and Weyl key schedule.
__host__ __device__ __forceinline__ uint4 philox4x32_10(uint4 c, uint32_t k0, uint32_t k1) {
#pragma unroll
    for (int r = 0; r < 10; ++r) {
#ifdef __CUDA_ARCH__
        const uint32_t lo0 = 0xD2511F53u * c.x, hi0 = __umulhi(0xD2511F53u, c.x);
        const uint32_t lo1 = 0xCD9E8D57u * c.z, hi1 = __umulhi(0xCD9E8D57u, c.z);
#else
        const uint64_t p0 = (uint64_t)0xD2511F53u * c.x, p1 = (uint64_t)0xCD9E8D57u * c.z;
        const uint32_t lo0 = (uint32_t)p0, hi0 = (uint32_t)(p0 >> 32);
        const uint32_t lo1 = (uint32_t)p1, hi1 = (uint32_t)(p1 >> 32);
#endif
        c = make_uint4(hi1 ^ c.y ^ k0, lo1, hi0 ^ c.w ^ k1, lo0);
        k0 += 0x9E3779B9u;
        k1 += 0xBB67AE85u;
    }
    return c;
}

// 24-bit uniform in (0,1), exactly the value the FP64 oracle uses.
__host__ __device__ __forceinline__ float u24(uint32_t x) { return fmaf((float)(x >> 8), 0x1p-24f, 0x1p-25f); }

#ifdef __CUDACC__
// Reflectance of an interface for incidence cosine ci (0 < ci <= 1) from index ni into nt:
// GetCriticalCos, ComputeTransmitCosine and ComputeFrenselReflectance of the reference
// (base/xmcml/xmcml/mcml_kernel.cpp:497-564, :644-661). Total internal reflection gives 1; within
// 1e-3 of the critical cosine the unpolarised Fresnel formula is evaluated in FP64.
__device__ __forceinline__ float fresnel_reflectance(float ni, float nt, float ci) {
    if (ni == nt) return 0.0f;
    const float cc = ni > nt ? sqrtf(1.0f - (nt * nt) / (ni * ni)) : 0.0f;
    if (ci <= cc) return 1.0f;
    if (ci > 1.0f - 1e-6f) {
        const float r = (nt - ni) / (nt + ni);
        return r * r;
    }
    if (ci < 1e-6f) return 1.0f;
    if (ni > nt && ci - cc < 1e-3f) {
        const double Ci = ci, Ni = ni, Nt = nt;
        const double Si = sqrt(1.0 - Ci * Ci);
        const double St = Ni * Si / Nt;
        if (St >= 1.0) return 1.0f;
        const double Ct = sqrt(1.0 - St * St);
        const double cs = Ci * Ct - Si * St, cd = Ci * Ct + Si * St;
        const double ss = Si * Ct + Ci * St, sd = Si * Ct - Ci * St;
        return (float)(0.5 * sd * sd * (cd * cd + cs * cs) / (ss * ss * cd * cd));
    }
    const float si = sqrtf(1.0f - ci * ci);
    const float st = ni * si / nt;
    if (st >= 1.0f) return 1.0f;
    const float ct = sqrtf(1.0f - st * st);
    const float cs = ci * ct - si * st, cd = ci * ct + si * st;
    const float ss = si * ct + ci * st, sd = si * ct - ci * st;
    return 0.5f * sd * sd * (cd * cd + cs * cs) / (ss * ss * cd * cd);
}

// GetNewPhotonDirection / ComputeCosineTheta (mcml_kernel.cpp:442-495): Henyey-Greenstein cos(theta)
// from u1 by the inverse CDF (hg_* = 1 - g^2, 1 + g^2, 1 / 2g, 1 - g, 2g; isotropic when hg_e == 0),
// azimuth 2 pi u2, and the rotation of (dx, dy, dz) with the near-vertical special case.
__device__ __forceinline__ void hg_spin(float hg_a, float hg_b, float hg_c, float hg_d, float hg_e, float u1, float u2,
                                        float& dx, float& dy, float& dz) {
    float cost;
    if (hg_e != 0.0f) {
        const float t = hg_a / (hg_d + hg_e * u1);
        cost = (hg_b - t * t) * hg_c;
    } else {
        cost = 2.0f * u1 - 1.0f;
    }
    cost = fminf(1.0f, fmaxf(-1.0f, cost));
    const float sint = sqrtf(fmaxf(0.0f, 1.0f - cost * cost));
    float a = u2;
    a = a > 0.5f ? a - 1.0f : a;  // same angle as 2*pi*u, reduced to [-pi, pi]
    float sp, cp;
    __sincosf(6.283185307179586f * a, &sp, &cp);
    const float ux = dx, uy = dy, uz = dz;
    const float rho2 = ux * ux + uy * uy;
    float nx, ny, nz;
    if (rho2 > 1e-12f) {
        const float irho = rsqrtf(rho2);
        const float rho = rho2 * irho;
        nx = sint * (ux * uz * cp - uy * sp) * irho + ux * cost;
        ny = sint * (uy * uz * cp + ux * sp) * irho + uy * cost;
        nz = -sint * cp * rho + uz * cost;
    } else {
        nx = sint * cp;
        ny = sint * sp;
        nz = uz >= 0.0f ? cost : -cost;
    }
    const float on = rsqrtf(nx * nx + ny * ny + nz * nz);
    dx = nx * on;
    dy = ny * on;
    dz = nz * on;
}
#endif

}  // namespace xmc
