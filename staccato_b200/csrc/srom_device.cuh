// Device-side building blocks shared by the sweep kernels.
//
// Rounding contract (shared bit-for-bit with oracle/srom_oracle.c): complex c - a*b is two
// fused multiply-adds per component, reciprocal and division use Smith's algorithm with
// separately rounded products, and the assembly follows the reference's three zaxpy passes
// (src/analysis/KrylovROMSubstructure.cpp:1411-1420) with every product and sum rounded on
// its own.  The explicit __fma_rn/__dmul_rn/__dadd_rn intrinsics stop the compiler from
// contracting or reassociating any of them.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

namespace srom {

constexpr unsigned FULL_MASK = 0xffffffffu;

// Device copy of one ROM descriptor (see srom_rom_desc in include/staccato_rom.h).
struct RomDev {
    int n, r, F, ldk;
    const double2 *K, *M, *D;
    double eta;
    const double2 *rhs;
    int ldb;
    const double *omega;
    double2 *X;
    int *info;
    int *steps;
    double *berr;
    double2 *LU;
    int *ipiv;
};

// One (ROM, frequency) system.
struct Item {
    int rom;
    int f;
};

// L2 policy for the ROM operators K, M, D: every frequency of a ROM (hence every CTA sweeping it)
// reads them, while each CTA's own scratch matrix streams through L2 once per panel step; marked
// evict-last they stay resident instead of being re-read from HBM by every CTA.
__device__ __forceinline__ uint64_t l2_keep_policy() {
    uint64_t p;
    asm("createpolicy.fractional.L2::evict_last.b64 %0, 1.0;" : "=l"(p));
    return p;
}

__device__ __forceinline__ double2 ld_keep(const double2 *ptr, uint64_t pol) {
    double2 v;
    asm("ld.global.L2::cache_hint.v2.f64 {%0, %1}, [%2], %3;" : "=d"(v.x), "=d"(v.y) : "l"(ptr), "l"(pol));
    return v;
}

__device__ __forceinline__ double2 csubmul(double2 c, double2 a, double2 b) {
    double2 o;
    o.x = __fma_rn(-a.x, b.x, __fma_rn(a.y, b.y, c.x));
    o.y = __fma_rn(-a.x, b.y, __fma_rn(-a.y, b.x, c.y));
    return o;
}

__device__ __forceinline__ double2 cmul(double2 a, double2 b) {
    double t0 = __dmul_rn(a.x, b.x), t1 = __dmul_rn(a.y, b.y);
    double t2 = __dmul_rn(a.x, b.y), t3 = __dmul_rn(a.y, b.x);
    return make_double2(__dsub_rn(t0, t1), __dadd_rn(t2, t3));
}

__device__ __forceinline__ double2 crecip(double2 z) {
    if (fabs(z.x) >= fabs(z.y)) {
        double t = __ddiv_rn(z.y, z.x);
        double d = __dadd_rn(z.x, __dmul_rn(z.y, t));
        return make_double2(__ddiv_rn(1.0, d), __ddiv_rn(-t, d));
    } else {
        double t = __ddiv_rn(z.x, z.y);
        double d = __dadd_rn(__dmul_rn(z.x, t), z.y);
        return make_double2(__ddiv_rn(t, d), __ddiv_rn(-1.0, d));
    }
}

__device__ __forceinline__ double2 cdiv(double2 a, double2 b) {
    if (fabs(b.x) >= fabs(b.y)) {
        double t = __ddiv_rn(b.y, b.x);
        double d = __dadd_rn(b.x, __dmul_rn(b.y, t));
        double re = __dadd_rn(a.x, __dmul_rn(a.y, t));
        double im = __dsub_rn(a.y, __dmul_rn(a.x, t));
        return make_double2(__ddiv_rn(re, d), __ddiv_rn(im, d));
    } else {
        double t = __ddiv_rn(b.x, b.y);
        double d = __dadd_rn(__dmul_rn(b.x, t), b.y);
        double re = __dadd_rn(__dmul_rn(a.x, t), a.y);
        double im = __dsub_rn(__dmul_rn(a.y, t), a.x);
        return make_double2(__ddiv_rn(re, d), __ddiv_rn(im, d));
    }
}

__device__ __forceinline__ double cabs1(double2 z) { return __dadd_rn(fabs(z.x), fabs(z.y)); }

// One entry of A(w) = (1 + i eta) K + (-w^2) M + (i w) D.  s = -(w*w).
__device__ __forceinline__ double2 assemble_entry(double2 k, double2 m, const double2 *D,
                                                  int64_t e, double eta, double s, double w) {
    if (eta != 0.0) {
        double t1 = __dmul_rn(eta, k.y), t2 = __dmul_rn(eta, k.x);
        k.x = __dsub_rn(k.x, t1);
        k.y = __dadd_rn(k.y, t2);
    }
    double2 v;
    v.x = __dadd_rn(k.x, __dmul_rn(s, m.x));
    v.y = __dadd_rn(k.y, __dmul_rn(s, m.y));
    if (D) {
        double2 d = D[e];
        v.x = __dsub_rn(v.x, __dmul_rn(w, d.y));
        v.y = __dadd_rn(v.y, __dmul_rn(w, d.x));
    }
    return v;
}

__device__ __forceinline__ void swap2(double2 &a, double2 &b) {
    double2 t = a;
    a = b;
    b = t;
}

}  // namespace srom

namespace srom {

// Complex arithmetic per storage type.  double2: the bit-exact FP64 contract above.
// float2: the mixed-precision factorisation (fused multiply-adds, Smith division).
template <typename T>
struct CT;

template <>
struct CT<double2> {
    using R = double;
    static __device__ __forceinline__ double2 subm(double2 c, double2 a, double2 b) { return csubmul(c, a, b); }
    // csubmul split into its two FMA layers (c.x += a.y b.y, c.y -= a.y b.x; then the a.x terms)
    static __device__ __forceinline__ void subm_first(double2 &c, double2 a, double2 b) {
        c.x = __fma_rn(a.y, b.y, c.x);
        c.y = __fma_rn(-a.y, b.x, c.y);
    }
    static __device__ __forceinline__ void subm_second(double2 &c, double2 a, double2 b) {
        c.x = __fma_rn(-a.x, b.x, c.x);
        c.y = __fma_rn(-a.x, b.y, c.y);
    }
    static __device__ __forceinline__ double2 mul(double2 a, double2 b) { return cmul(a, b); }
    static __device__ __forceinline__ double2 recip(double2 z) { return crecip(z); }
    static __device__ __forceinline__ double2 div(double2 a, double2 b) { return cdiv(a, b); }
    static __device__ __forceinline__ double abs1(double2 z) { return cabs1(z); }
    static __device__ __forceinline__ double2 zero() { return make_double2(0.0, 0.0); }
    static __device__ __forceinline__ double2 shfl(double2 v, int src, int width) {
        return make_double2(__shfl_sync(FULL_MASK, v.x, src, width), __shfl_sync(FULL_MASK, v.y, src, width));
    }
};

template <>
struct CT<float2> {
    using R = float;
    static __device__ __forceinline__ float2 subm(float2 c, float2 a, float2 b) {
        return make_float2(__fmaf_rn(-a.x, b.x, __fmaf_rn(a.y, b.y, c.x)),
                           __fmaf_rn(-a.x, b.y, __fmaf_rn(-a.y, b.x, c.y)));
    }
    static __device__ __forceinline__ float2 mul(float2 a, float2 b) {
        return make_float2(__fmaf_rn(a.x, b.x, -a.y * b.y), __fmaf_rn(a.x, b.y, a.y * b.x));
    }
    static __device__ __forceinline__ void subm_first(float2 &c, float2 a, float2 b) {
        c.x = __fmaf_rn(a.y, b.y, c.x);
        c.y = __fmaf_rn(-a.y, b.x, c.y);
    }
    static __device__ __forceinline__ void subm_second(float2 &c, float2 a, float2 b) {
        c.x = __fmaf_rn(-a.x, b.x, c.x);
        c.y = __fmaf_rn(-a.x, b.y, c.y);
    }
    static __device__ __forceinline__ float2 recip(float2 z) {
        if (fabsf(z.x) >= fabsf(z.y)) {
            float t = z.y / z.x, d = z.x + z.y * t;
            return make_float2(1.0f / d, -t / d);
        }
        float t = z.x / z.y, d = z.x * t + z.y;
        return make_float2(t / d, -1.0f / d);
    }
    static __device__ __forceinline__ float2 div(float2 a, float2 b) {
        if (fabsf(b.x) >= fabsf(b.y)) {
            float t = b.y / b.x, d = b.x + b.y * t;
            return make_float2((a.x + a.y * t) / d, (a.y - a.x * t) / d);
        }
        float t = b.x / b.y, d = b.x * t + b.y;
        return make_float2((a.x * t + a.y) / d, (a.y * t - a.x) / d);
    }
    static __device__ __forceinline__ float abs1(float2 z) { return fabsf(z.x) + fabsf(z.y); }
    static __device__ __forceinline__ float2 zero() { return make_float2(0.f, 0.f); }
    static __device__ __forceinline__ float2 shfl(float2 v, int src, int width) {
        return make_float2(__shfl_sync(FULL_MASK, v.x, src, width), __shfl_sync(FULL_MASK, v.y, src, width));
    }
};

}  // namespace srom
