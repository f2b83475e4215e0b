// nf_pair.cuh -- per-pair softened gravity on the B200 FP32 pipe.
//
// Softening formulas follow singlestep/Direct/DirectGPUKernels.cuh:20-174
// (Plummer :144-174, single spline :68-108, cubic spline :20-66, cubic
// Plummer :110-143).  Differences from the reference GPU kernel, all in the
// direction of accuracy:
//   * rsqrt is the hardware estimate (rsqrt.approx.ftz.f32) followed by one
//     Newton-Raphson step; for the far field the step is applied to the cube:
//       y = rsqrt(r2); e = r2*y^2 - 1; r2^-3/2 ~= y^3 * (1 - 1.5 e)
//     (first-order Newton correction of y, cubed: 5 FP32 instructions).
//   * the single spline is accumulated in far units, g = f_ref / eps^3
//     (r^-3 in the far branch), and the sum is multiplied by eps^3 once per
//     sink.  Source cells that cannot hold a pair closer than one cell width
//     use the far branch alone; cells adjacent to the sink's cell evaluate
//     both branches (spline_g_both).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

namespace nf {

enum { SOFT_PLUMMER = 0, SOFT_SINGLE_SPLINE = 1, SOFT_CUBIC_SPLINE = 2, SOFT_CUBIC_PLUMMER = 3 };

// Hardware reciprocal square root estimate (one MUFU.RSQ).
__device__ __forceinline__ float rsqrt_est(float x) {
    float y;
    asm("rsqrt.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
    return y;
}

// r2^-3/2 from the estimate plus one Newton step on the cube.
__device__ __forceinline__ float inv_r3(float r2) {
    float y = rsqrt_est(r2);
    float y2 = y * y;
    float y3 = y2 * y;
    float e = fmaf(r2, y2, -1.0f);
    float g = y3 * e;
    return fmaf(g, -1.5f, y3);
}

// rsqrt with one Newton step: y (1.5 - 0.5 x y^2).
__device__ __forceinline__ float rsqrt_nr(float x) {
    float y = rsqrt_est(x);
    float h = x * y;
    float e = fmaf(-h, y, 1.0f);
    return fmaf(0.5f * y, e, y);
}

// TwoSum (Knuth): s + err == a + b exactly.
__device__ __forceinline__ void two_sum(float a, float b, float &s, float &err) {
    s = a + b;
    float bb = s - a;
    err = (a - (s - bb)) + (b - bb);
}

// Kernel constants shared by every pair of a launch.
struct PairConst {
    float eps;        // the reference kernel parameter (eps^2, 1/eps^2, 1/eps, eps^3)
    float near_thr;   // single spline: eps^2 (unscaled)
    float inv_eps3;   // single spline: eps^-3
    float b2;         // FOF density radius^2 (0 = off)
    // single spline near branch in far units (g = f_ref / eps^3):
    //   (-15 u + 6 u^2 + 10) / eps^3 with u = r/eps = r^2 y / eps
    //   = (c1 y + c2) r^2 + c3,  c1 = -15 eps^-4, c2 = 6 eps^-5, c3 = 10 eps^-3
    float c1, c2, c3;
};

// Default evaluation: returns g with a -= g * d.
// Plummer: (r^2 + eps^2)^-3/2.  Single spline far branch: r^-3 (r^2 floored
// at 1e-25, far below any eps^2, so that a zero separation stays finite).
template <int SOFT>
__device__ __forceinline__ float pair_g_fast(float dx, float dy, float dz, const PairConst &pc,
                                             float &r2_out) {
    if (SOFT == SOFT_PLUMMER) {
        float r2 = fmaf(dz, dz, fmaf(dy, dy, fmaf(dx, dx, pc.eps)));
        r2_out = r2;
        return inv_r3(r2);
    } else if (SOFT == SOFT_SINGLE_SPLINE) {
        float r2 = fmaf(dz, dz, fmaf(dy, dy, fmaf(dx, dx, 1e-25f)));
        r2_out = r2;
        return inv_r3(r2);
    } else if (SOFT == SOFT_CUBIC_SPLINE) {
        // Hernquist & Katz cubic spline, DirectGPUKernels.cuh:31-65.
        float r2 = fmaf(dz, dz, fmaf(dy, dy, fmaf(dx, dx, 1e-30f)));
        r2_out = r2;
        float rinv = rsqrt_nr(r2);
        float u = pc.eps / rinv;
        float r3 = rinv * rinv * rinv;
        float spf;
        if (u >= 2.0f) {
            spf = r3;
        } else if (u >= 1.0f) {
            float u3 = u * u * u;
            spf = r3 * (-1.0f / 15.0f + (8.0f / 3.0f) * u3 - 3.0f * u3 * u +
                        (6.0f / 5.0f) * u3 * u * u - (1.0f / 6.0f) * u3 * u3);
        } else {
            float ei3 = pc.eps * pc.eps * pc.eps;
            spf = ei3 * ((4.0f / 3.0f) - (6.0f / 5.0f) * u * u + 0.5f * u * u * u);
        }
        return spf;
    } else {
        // cubic Plummer, DirectGPUKernels.cuh:124-143 (TAU2 = 1e-16).
        float r = fmaf(dz, dz, fmaf(dy, dy, fmaf(dx, dx, 1e-16f)));
        r2_out = r;
        float r3 = r * r * rsqrt_nr(r);
        return 1.0f / (r3 + pc.eps);
    }
}

// Single spline, both branches, for source cells adjacent to the sink cell
// (the only ones that can hold pairs closer than eps).  The reference writes
// it as min(f^3, (-15 f + 6) dr2 + 10) in eps units (DirectCPUKernels.cc:71;
// the GPU's branch on dr2 > 1, DirectGPUKernels.cuh:94-98, selects the same
// value because the two branches touch to second order at u = 1 and the
// polynomial is the smaller one for u < 1).  Here it is evaluated in far
// units with the Newton-corrected y = 1/r:
//   g = min(y^3, (c1 y + c2) r^2 + c3)
// A self pair (d = 0, r^2 = 1e-25 floor) gives a finite g times d = 0; a
// padding record far away gives an infinite polynomial and g ~ 0.
__device__ __forceinline__ float spline_g_both(float dx, float dy, float dz,
                                               const PairConst &pc) {
    float r2 = fmaf(dz, dz, fmaf(dy, dy, fmaf(dx, dx, 1e-25f)));
    float y = rsqrt_est(r2);
    float y2 = y * y;
    float e = fmaf(r2, y2, -1.0f);
    float yn = fmaf(-0.5f * e, y, y);
    float gfar = yn * yn * yn;
    float gnear = fmaf(fmaf(pc.c1, yn, pc.c2), r2, pc.c3);
    return fminf(gfar, gnear);
}

// ---------------------------------------------------------------------------
// Two sinks per instruction.  sm_100 executes FP32 add/mul/fma on register
// pairs (f32x2): one issue slot for two results, the same per-component
// rounding as the scalar instruction.  The pair loop is issue-bound in
// scalar form (~15 issue slots per pair against 14 FP32 results), so pairing
// the sinks of a lane moves the bound to the FP32 pipe itself.  Each helper
// below is the component-wise twin of the scalar code above, operation for
// operation, so a paired evaluation is bit-identical to the scalar one.
// ---------------------------------------------------------------------------
__device__ __forceinline__ float2 add2(float2 a, float2 b) { return __fadd2_rn(a, b); }
__device__ __forceinline__ float2 mul2(float2 a, float2 b) { return __fmul2_rn(a, b); }
__device__ __forceinline__ float2 fma2(float2 a, float2 b, float2 c) { return __ffma2_rn(a, b, c); }
__device__ __forceinline__ float2 dup2(float v) { return make_float2(v, v); }

// inv_r3 on a pair.
__device__ __forceinline__ float2 inv_r3_x2(float2 r2) {
    float2 y = make_float2(rsqrt_est(r2.x), rsqrt_est(r2.y));
    float2 y2 = mul2(y, y);
    float2 y3 = mul2(y2, y);
    float2 e = fma2(r2, y2, dup2(-1.0f));
    float2 g = mul2(y3, e);
    return fma2(g, dup2(-1.5f), y3);
}

// r^2 (+ the kernel's additive constant a2) of a pair of separations.
__device__ __forceinline__ float2 r2_x2(float2 dx, float2 dy, float2 dz, float a2) {
    return fma2(dz, dz, fma2(dy, dy, fma2(dx, dx, dup2(a2))));
}

// spline_g_both on a pair (r2 already floored by its 1e-25 addend).
__device__ __forceinline__ float2 spline_g_both_x2(float2 r2, const PairConst &pc) {
    float2 y = make_float2(rsqrt_est(r2.x), rsqrt_est(r2.y));
    float2 y2 = mul2(y, y);
    float2 e = fma2(r2, y2, dup2(-1.0f));
    float2 yn = fma2(mul2(dup2(-0.5f), e), y, y);
    float2 gfar = mul2(mul2(yn, yn), yn);
    float2 gnear = fma2(fma2(dup2(pc.c1), yn, dup2(pc.c2)), r2, dup2(pc.c3));
    return make_float2(fminf(gfar.x, gnear.x), fminf(gfar.y, gnear.y));
}

// Unsoftened r^2 for the FOF density sum (w += b2 - r^2 if r^2 < b2).
__device__ __forceinline__ float dens_term(float dx, float dy, float dz, float b2) {
    float r2 = fmaf(dz, dz, fmaf(dy, dy, dx * dx));
    return r2 < b2 ? b2 - r2 : 0.0f;
}

}  // namespace nf
