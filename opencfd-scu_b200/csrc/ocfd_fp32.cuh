// ocfd_fp32.cuh -- single-precision point formulas of the precision form
// (sm_100a).
//
// Overloads, by argument type, of the FP64 point formulas in
// ocfd_device.cuh and ocfd_face.cuh: the same schemes restated in FP32 so
// that a kernel templated on its real type picks them up unchanged.  They
// are not bit-for-bit images of the FP64 formulas (that is not their
// purpose): the WENO weights are formed as d_k / (eps + beta_k)^2, which is
// the reference's d_k * prod_{j != k} (eps + beta_j)^2 divided through by
// the product of all four (five for WENO5), so that no product of squared
// smoothness indicators can leave the FP32 range across a strong jump.
// The FP64 path keeps the reference's form.
#pragma once
#include "ocfd_face.cuh"

namespace ocfd {

// FP32 quotients and square roots stay correctly rounded: the hardware
// approximations (__fdividef, x * rsqrtf(x)) were measured to let a
// curvilinear shock case drift from 1e-7 to 3e-4 relative to FP64 within
// ten steps.  Division by a run-time constant is a product with its
// reciprocal (div_const below).
__device__ __forceinline__ float sqrt_r(float x) { return sqrtf(x); }
__device__ __forceinline__ double sqrt_r(double x) { return sqrt(x); }
__device__ __forceinline__ float fdiv(float a, float b) { return a / b; }

// the LAP-box primitives and the stage RHS in the precision of a kernel
template <typename R> __device__ __forceinline__ const R *prim_r(const Params &p, int m);
template <> __device__ __forceinline__ const double *prim_r<double>(const Params &p, int m) { return p.prim[m]; }
template <> __device__ __forceinline__ const float *prim_r<float>(const Params &p, int m) { return p.prim32[m]; }
template <typename D> __device__ __forceinline__ D *du_r(const Params &p);
template <> __device__ __forceinline__ double *du_r<double>(const Params &p) { return p.du; }
template <> __device__ __forceinline__ float *du_r<float>(const Params &p) { return p.du32; }
template <typename R> __device__ __forceinline__ R *ev_r(const Params &p);
template <> __device__ __forceinline__ double *ev_r<double>(const Params &p) { return p.ev; }
template <> __device__ __forceinline__ float *ev_r<float>(const Params &p) { return p.ev32; }

__device__ __forceinline__ float div_const(float x, float c, float inv) { return x * inv; }

// Steger-Warming split with the direction's |A| and A/|A| already formed
template <bool EPS0>
__device__ __forceinline__ void sw_split_pre(float tmp0, float u, float v, float w, float cc,
                                             float A1, float A2, float A3, float ss,
                                             float An1, float An2, float An3,
                                             const Params &p, float *fp, float *fm) {
    const float eps = (float)p.epsl_sw, G = (float)p.Gamma;
    float E1 = A1 * u + A2 * v + A3 * w;
    float E2 = E1 - cc * ss;
    float E3 = E1 + cc * ss;
    float E1P = (E1 + (EPS0 ? fabsf(E1) : sqrtf(E1 * E1 + eps * eps))) * 0.5f;
    float E2P = (E2 + (EPS0 ? fabsf(E2) : sqrtf(E2 * E2 + eps * eps))) * 0.5f;
    float E3P = (E3 + (EPS0 ? fabsf(E3) : sqrtf(E3 * E3 + eps * eps))) * 0.5f;
    float E1M = E1 - E1P, E2M = E2 - E2P, E3M = E3 - E3P;
    float uc1 = u - cc * An1, uc2 = u + cc * An1;
    float vc1 = v - cc * An2, vc2 = v + cc * An2;
    float wc1 = w - cc * An3, wc2 = w + cc * An3;
    float vvc1 = (uc1 * uc1 + vc1 * vc1 + wc1 * wc1) * 0.5f;
    float vvc2 = (uc2 * uc2 + vc2 * vc2 + wc2 * wc2) * 0.5f;
    float vv = (G - 1.0f) * (u * u + v * v + w * w);
    float W2 = (float)p.split_C3 * cc * cc;
    const float C1 = (float)p.split_C1;
    fp[0] = tmp0 * (C1 * E1P + E2P + E3P);
    fp[1] = tmp0 * (C1 * E1P * u + E2P * uc1 + E3P * uc2);
    fp[2] = tmp0 * (C1 * E1P * v + E2P * vc1 + E3P * vc2);
    fp[3] = tmp0 * (C1 * E1P * w + E2P * wc1 + E3P * wc2);
    fp[4] = tmp0 * (E1P * vv + E2P * vvc1 + E3P * vvc2 + W2 * (E2P + E3P));
    fm[0] = tmp0 * (C1 * E1M + E2M + E3M);
    fm[1] = tmp0 * (C1 * E1M * u + E2M * uc1 + E3M * uc2);
    fm[2] = tmp0 * (C1 * E1M * v + E2M * vc1 + E3M * vc2);
    fm[3] = tmp0 * (C1 * E1M * w + E2M * wc1 + E3M * wc2);
    fm[4] = tmp0 * (E1M * vv + E2M * vvc1 + E3M * vvc2 + W2 * (E2M + E3M));
}

// the same from the metric row of the point (curvilinear grids)
__device__ __forceinline__ void sw_split(float tmp0, float u, float v, float w, float cc,
                                         float A1, float A2, float A3, float G, float eps,
                                         float split_C1, float split_C3, float *fp, float *fm) {
    float ss = sqrtf(A1 * A1 + A2 * A2 + A3 * A3);
    float E1 = A1 * u + A2 * v + A3 * w;
    float E2 = E1 - cc * ss;
    float E3 = E1 + cc * ss;
    ss = 1.0f / ss;
    A1 *= ss; A2 *= ss; A3 *= ss;
    float E1P = (E1 + sqrtf(E1 * E1 + eps * eps)) * 0.5f;
    float E2P = (E2 + sqrtf(E2 * E2 + eps * eps)) * 0.5f;
    float E3P = (E3 + sqrtf(E3 * E3 + eps * eps)) * 0.5f;
    float E1M = E1 - E1P, E2M = E2 - E2P, E3M = E3 - E3P;
    float uc1 = u - cc * A1, uc2 = u + cc * A1;
    float vc1 = v - cc * A2, vc2 = v + cc * A2;
    float wc1 = w - cc * A3, wc2 = w + cc * A3;
    float vvc1 = (uc1 * uc1 + vc1 * vc1 + wc1 * wc1) * 0.5f;
    float vvc2 = (uc2 * uc2 + vc2 * vc2 + wc2 * wc2) * 0.5f;
    float vv = (G - 1.0f) * (u * u + v * v + w * w);
    float W2 = split_C3 * cc * cc;
    fp[0] = tmp0 * (split_C1 * E1P + E2P + E3P);
    fp[1] = tmp0 * (split_C1 * E1P * u + E2P * uc1 + E3P * uc2);
    fp[2] = tmp0 * (split_C1 * E1P * v + E2P * vc1 + E3P * vc2);
    fp[3] = tmp0 * (split_C1 * E1P * w + E2P * wc1 + E3P * wc2);
    fp[4] = tmp0 * (E1P * vv + E2P * vvc1 + E3P * vvc2 + W2 * (E2P + E3P));
    fm[0] = tmp0 * (split_C1 * E1M + E2M + E3M);
    fm[1] = tmp0 * (split_C1 * E1M * u + E2M * uc1 + E3M * uc2);
    fm[2] = tmp0 * (split_C1 * E1M * v + E2M * vc1 + E3M * vc2);
    fm[3] = tmp0 * (split_C1 * E1M * w + E2M * wc1 + E3M * wc2);
    fm[4] = tmp0 * (E1M * vv + E2M * vvc1 + E3M * vvc2 + W2 * (E2M + E3M));
}

// UP7 with the /420 as a corrected product
__device__ __forceinline__ float up7_p_q(const float *s) {
    return div_const(-3.0f*s[0] + 25.0f*s[1] - 101.0f*s[2] + 319.0f*s[3] + 214.0f*s[4]
                     - 38.0f*s[5] + 4.0f*s[6], 420.0f, 1.0f / 420.0f);
}
__device__ __forceinline__ float up7_m_q(const float *s) {
    return div_const(-3.0f*s[7] + 25.0f*s[6] - 101.0f*s[5] + 319.0f*s[4] + 214.0f*s[3]
                     - 38.0f*s[2] + 4.0f*s[1], 420.0f, 1.0f / 420.0f);
}

// WENO7 smoothness indicator of the 4-point sub-stencil q[0..3] written as
// in the reference (the 960 / 1040 / 1043 / 80 form, first/second/third
// differences t, t1, t2), for sub-stencil index k
__device__ __forceinline__ float w7_beta(float t, float t1, float t2) {
    return 960.0f*t*t + 1040.0f*t1*t1 + 1043.0f*t2*t2 + 80.0f*(t*t2);
}

// WENO7, s[0..6] = f(F-3..F+3) (positive side)
__device__ __forceinline__ float weno7_p(const float *s) {
    const float S0 = w7_beta(-2.0f*s[0] + 9.0f*s[1] - 18.0f*s[2] + 11.0f*s[3],
                             -6.0f*s[0] + 24.0f*s[1] - 30.0f*s[2] + 12.0f*s[3],
                             -6.0f*s[0] + 18.0f*(s[1] - s[2]) + 6.0f*s[3]);
    const float S1 = w7_beta(s[1] - 6.0f*s[2] + 3.0f*s[3] + 2.0f*s[4],
                             6.0f*s[2] - 12.0f*s[3] + 6.0f*s[4],
                             -6.0f*s[1] + 18.0f*(s[2] - s[3]) + 6.0f*s[4]);
    const float S2 = w7_beta(-2.0f*s[2] - 3.0f*s[3] + 6.0f*s[4] - s[5],
                             6.0f*s[3] - 12.0f*s[4] + 6.0f*s[5],
                             -6.0f*s[2] + 18.0f*(s[3] - s[4]) + 6.0f*s[5]);
    const float S3 = w7_beta(-11.0f*s[3] + 18.0f*s[4] - 9.0f*s[5] + 2.0f*s[6],
                             12.0f*s[3] - 30.0f*s[4] + 24.0f*s[5] - 6.0f*s[6],
                             -6.0f*s[3] + 18.0f*(s[4] - s[5]) + 6.0f*s[6]);
    const float e = 3.456e-4f;
    const float a0 = fdiv(1.0f, (e + S0) * (e + S0)), a1 = fdiv(12.0f, (e + S1) * (e + S1));
    const float a2 = fdiv(18.0f, (e + S2) * (e + S2)), a3 = fdiv(4.0f, (e + S3) * (e + S3));
    const float r = a0 * (-3.0f*s[0] + 13.0f*s[1] - 23.0f*s[2] + 25.0f*s[3])
                  + a1 * (s[1] - 5.0f*s[2] + 13.0f*s[3] + 3.0f*s[4])
                  + a2 * (-s[2] + 7.0f*s[3] + 7.0f*s[4] - s[5])
                  + a3 * (3.0f*s[3] + 13.0f*s[4] - 5.0f*s[5] + s[6]);
    return fdiv(r, 12.0f * (a0 + a1 + a2 + a3));
}

// WENO7 negative side, s8[1..7] = f(F-2..F+4)
__device__ __forceinline__ float weno7_m(const float *s8) {
    const float *s = s8 + 1;
    const float S0 = w7_beta(-2.0f*s[6] + 9.0f*s[5] - 18.0f*s[4] + 11.0f*s[3],
                             -6.0f*s[6] + 24.0f*s[5] - 30.0f*s[4] + 12.0f*s[3],
                             -6.0f*s[6] + 18.0f*(s[5] - s[4]) + 6.0f*s[3]);
    const float S1 = w7_beta(s[5] - 6.0f*s[4] + 3.0f*s[3] + 2.0f*s[2],
                             6.0f*s[4] - 12.0f*s[3] + 6.0f*s[2],
                             -6.0f*s[5] + 18.0f*(s[4] - s[3]) + 6.0f*s[2]);
    const float S2 = w7_beta(-2.0f*s[4] - 3.0f*s[3] + 6.0f*s[2] - s[1],
                             6.0f*s[3] - 12.0f*s[2] + 6.0f*s[1],
                             -6.0f*s[4] + 18.0f*(s[3] - s[2]) + 6.0f*s[1]);
    const float S3 = w7_beta(-11.0f*s[3] + 18.0f*s[2] - 9.0f*s[1] + 2.0f*s[0],
                             12.0f*s[3] - 30.0f*s[2] + 24.0f*s[1] - 6.0f*s[0],
                             -6.0f*s[3] + 18.0f*(s[2] - s[1]) + 6.0f*s[0]);
    const float e = 3.456e-4f;
    const float a0 = fdiv(1.0f, (e + S0) * (e + S0)), a1 = fdiv(12.0f, (e + S1) * (e + S1));
    const float a2 = fdiv(18.0f, (e + S2) * (e + S2)), a3 = fdiv(4.0f, (e + S3) * (e + S3));
    const float r = a0 * (-3.0f*s[6] + 13.0f*s[5] - 23.0f*s[4] + 25.0f*s[3])
                  + a1 * (s[5] - 5.0f*s[4] + 13.0f*s[3] + 3.0f*s[2])
                  + a2 * (-s[4] + 7.0f*s[3] + 7.0f*s[2] - s[1])
                  + a3 * (3.0f*s[3] + 13.0f*s[2] - 5.0f*s[1] + s[0]);
    return fdiv(r, 12.0f * (a0 + a1 + a2 + a3));
}

// WENO5 (positive side uses s8[1..5], negative side s8[2..6])
__device__ __forceinline__ float weno5_p(const float *s8) {
    const float *s = s8 + 1;
    const float ep = 1e-6f;
    float t = s[2] - 2.0f*s[3] + s[4], u = 3.0f*s[2] - 4.0f*s[3] + s[4];
    const float S0 = 13.0f*t*t + 3.0f*u*u;
    t = s[1] - 2.0f*s[2] + s[3]; u = s[1] - s[3];
    const float S1 = 13.0f*t*t + 3.0f*u*u;
    t = s[0] - 2.0f*s[1] + s[2]; u = s[0] - 4.0f*s[1] + 3.0f*s[2];
    const float S2 = 13.0f*t*t + 3.0f*u*u;
    const float a0 = fdiv(3.0f, (12.0f*ep + S0) * (12.0f*ep + S0));
    const float a1 = fdiv(6.0f, (12.0f*ep + S1) * (12.0f*ep + S1));
    const float a2 = fdiv(1.0f, (12.0f*ep + S2) * (12.0f*ep + S2));
    const float q03 = 2.0f*s[2] + 5.0f*s[3] - s[4];
    const float q13 = -s[1] + 5.0f*s[2] + 2.0f*s[3];
    const float q23 = 2.0f*s[0] - 7.0f*s[1] + 11.0f*s[2];
    return fdiv(a0*q03 + a1*q13 + a2*q23, 6.0f*(a0 + a1 + a2));
}
__device__ __forceinline__ float weno5_m(const float *s8) {
    const float *s = s8 + 2;
    const float ep = 1e-6f;
    float t = s[2] - 2.0f*s[1] + s[0], u = 3.0f*s[2] - 4.0f*s[1] + s[0];
    const float S0 = 13.0f*t*t + 3.0f*u*u;
    t = s[3] - 2.0f*s[2] + s[1]; u = s[3] - s[1];
    const float S1 = 13.0f*t*t + 3.0f*u*u;
    t = s[4] - 2.0f*s[3] + s[2]; u = s[4] - 4.0f*s[3] + 3.0f*s[2];
    const float S2 = 13.0f*t*t + 3.0f*u*u;
    const float a0 = fdiv(3.0f, (12.0f*ep + S0) * (12.0f*ep + S0));
    const float a1 = fdiv(6.0f, (12.0f*ep + S1) * (12.0f*ep + S1));
    const float a2 = fdiv(1.0f, (12.0f*ep + S2) * (12.0f*ep + S2));
    const float q03 = 2.0f*s[2] + 5.0f*s[1] - s[0];
    const float q13 = -s[3] + 5.0f*s[2] + 2.0f*s[1];
    const float q23 = 2.0f*s[4] - 7.0f*s[3] + 11.0f*s[2];
    return fdiv(a0*q03 + a1*q13 + a2*q23, 6.0f*(a0 + a1 + a2));
}

__device__ __forceinline__ float sgn1(float x2) { return x2 >= 0 ? 1.0f : -1.0f; }
__device__ __forceinline__ float minmod2(float x1, float x2) {
    return 0.5f*(sgn1(x1) + sgn1(x2))*fminf(fabsf(x1), fabsf(x2));
}

// one-sided WENO5 candidates of the boundary closures; s[0..4] = f(i-2..i+2)
__device__ __forceinline__ float w5_beta(float t, float u) { return 13.0f*t*t + 3.0f*u*u; }
// single-candidate closures: the candidate's weight cancels
__device__ __forceinline__ float w5_p_left(const float *s) {
    return (2.0f*s[2] + 5.0f*s[3] - s[4]) / 6.0f;
}
__device__ __forceinline__ float w5_m_left(const float *s) {
    return (2.0f*s[4] - 7.0f*s[3] + 11.0f*s[2]) / 6.0f;
}
__device__ __forceinline__ float w5_pair(float a, float qa, float b, float qb) {
    return (a*qa + b*qb) / (6.0f*(a + b));
}
__device__ __forceinline__ float w5_p_right_plus(const float *s) {
    const float ep12 = 12.0e-6f;
    const float S1 = w5_beta(s[1] - 2.0f*s[2] + s[3], s[1] - s[3]);
    const float S2 = w5_beta(s[0] - 2.0f*s[1] + s[2], s[0] - 4.0f*s[1] + 3.0f*s[2]);
    return w5_pair(6.0f / ((ep12 + S1)*(ep12 + S1)), -s[1] + 5.0f*s[2] + 2.0f*s[3],
                   1.0f / ((ep12 + S2)*(ep12 + S2)), 2.0f*s[0] - 7.0f*s[1] + 11.0f*s[2]);
}
__device__ __forceinline__ float w5_p_left_plus(const float *s) {
    const float ep12 = 12.0e-6f;
    const float S0 = w5_beta(s[2] - 2.0f*s[3] + s[4], 3.0f*s[2] - 4.0f*s[3] + s[4]);
    const float S1 = w5_beta(s[1] - 2.0f*s[2] + s[3], s[1] - s[3]);
    return w5_pair(3.0f / ((ep12 + S0)*(ep12 + S0)), 2.0f*s[2] + 5.0f*s[3] - s[4],
                   6.0f / ((ep12 + S1)*(ep12 + S1)), -s[1] + 5.0f*s[2] + 2.0f*s[3]);
}
__device__ __forceinline__ float w5_m_right_plus(const float *s) {
    const float ep12 = 12.0e-6f;
    const float S0 = w5_beta(s[2] - 2.0f*s[1] + s[0], 3.0f*s[2] - 4.0f*s[1] + s[0]);
    const float S1 = w5_beta(s[3] - 2.0f*s[2] + s[1], s[3] - s[1]);
    return w5_pair(3.0f / ((ep12 + S0)*(ep12 + S0)), 2.0f*s[2] + 5.0f*s[1] - s[0],
                   6.0f / ((ep12 + S1)*(ep12 + S1)), -s[3] + 5.0f*s[2] + 2.0f*s[1]);
}
__device__ __forceinline__ float w5_m_left_plus(const float *s) {
    const float ep12 = 12.0e-6f;
    const float S1 = w5_beta(s[3] - 2.0f*s[2] + s[1], s[3] - s[1]);
    const float S2 = w5_beta(s[4] - 2.0f*s[3] + s[2], s[4] - 4.0f*s[3] + 3.0f*s[2]);
    return w5_pair(6.0f / ((ep12 + S1)*(ep12 + S1)), -s[3] + 5.0f*s[2] + 2.0f*s[1],
                   1.0f / ((ep12 + S2)*(ep12 + S2)), 2.0f*s[4] - 7.0f*s[3] + 11.0f*s[2]);
}

// boundary closure of face F+1/2 (the FP64 closure() with these candidates)
__device__ __forceinline__ bool closure(int sign, bool lo, bool hi, int KA, int KB, int F, int n,
                                        const float *v, float &out) {
    int c = F + 1;
    if (sign == 0) {
        if (lo && c <= KA) {
            if (c == 0) out = v[4];
            else if (c == 1) out = w5_p_left(v + 1);
            else if (c == 2) out = w5_p_left_plus(v + 1);
            else out = weno5_p(v);
            return true;
        }
        if (hi) {
            int t = c - (n + 1);
            if (t >= -KB) {
                if (t == -1) out = v[3] + 0.5f * minmod2(v[3] - v[2], v[3] - v[2]);
                else if (t == -2) out = w5_p_right_plus(v + 1);
                else out = weno5_p(v);
                return true;
            }
        }
        return false;
    }
    if (lo && c < KA) {
        if (c == 0) out = w5_m_left(v + 2);
        else if (c == 1) out = w5_m_left_plus(v + 2);
        else out = weno5_m(v);
        return true;
    }
    if (hi) {
        int t = c - (n + 1);
        if (t >= -KB - 1) {
            if (t == -1) out = v[3];
            else if (t == -2) out = v[4] - 0.5f * minmod2(v[4] - v[3], v[4] - v[3]);
            else if (t == -3) out = w5_m_right_plus(v + 2);
            else out = weno5_m(v);
            return true;
        }
    }
    return false;
}

// characteristic eigen-rows from a face record in FP32 (layout of FP_N)
__device__ __forceinline__ void L_row(const float *r, int nf, int c, float S[5]) {
    const float u1 = r[FU * nf], v1 = r[FV * nf], w1 = r[FW * nf], KK = r[FKK * nf];
    switch (c) {
    case 0: S[0] = 1.0f - KK * r[FV2 * nf]; S[1] = KK * u1; S[2] = KK * v1; S[3] = KK * w1; S[4] = -KK; break;
    case 1: {
        float l1 = r[FL1 * nf], l2 = r[FL2 * nf], l3 = r[FL3 * nf];
        S[0] = -(u1 * l1 + v1 * l2 + w1 * l3); S[1] = l1; S[2] = l2; S[3] = l3; S[4] = 0.0f; break; }
    case 2: {
        float m1 = r[FM1 * nf], m2 = r[FM2 * nf], m3 = r[FM3 * nf];
        float n1 = r[FN1 * nf], n2 = r[FN2 * nf], n3 = r[FN3 * nf];
        float l1 = r[FL1 * nf], l2 = r[FL2 * nf], l3 = r[FL3 * nf];
        S[0] = -(u1 * m1 + v1 * m2 + w1 * m3);
        S[1] = n2 * l3 - n3 * l2; S[2] = n3 * l1 - n1 * l3; S[3] = n1 * l2 - n2 * l1; S[4] = 0.0f; break; }
    default: {
        float X1 = r[FX1 * nf], un = r[FUN * nf], v2 = r[FV2 * nf];
        float n1 = r[FN1 * nf], n2 = r[FN2 * nf], n3 = r[FN3 * nf];
        float s41 = KK * v2 * 0.5f + X1 * un;
        float s42 = -X1 * n1 - KK * u1 * 0.5f;
        float s43 = -X1 * n2 - KK * v1 * 0.5f;
        float s44 = -X1 * n3 - KK * w1 * 0.5f;
        if (c == 3) { S[0] = s41; S[1] = s42; S[2] = s43; S[3] = s44; S[4] = KK * 0.5f; }
        else { S[0] = s41 - 2 * X1 * un; S[1] = 2 * X1 * n1 + s42; S[2] = 2 * X1 * n2 + s43;
               S[3] = 2 * X1 * n3 + s44; S[4] = KK * 0.5f; }
        break; }
    }
}

__device__ __forceinline__ void R_col(const float *r, int nf, int c, float S[5]) {
    const float u1 = r[FU * nf], v1 = r[FV * nf], w1 = r[FW * nf], c1 = r[FC * nf];
    switch (c) {
    case 0: S[0] = 1.0f; S[1] = u1; S[2] = v1; S[3] = w1; S[4] = r[FV2 * nf]; break;
    case 1: { float l1 = r[FL1 * nf], l2 = r[FL2 * nf], l3 = r[FL3 * nf];
        S[0] = 0.0f; S[1] = l1; S[2] = l2; S[3] = l3; S[4] = u1 * l1 + v1 * l2 + w1 * l3; break; }
    case 2: { float n1 = r[FN1 * nf], n2 = r[FN2 * nf], n3 = r[FN3 * nf];
        float l1 = r[FL1 * nf], l2 = r[FL2 * nf], l3 = r[FL3 * nf];
        S[0] = 0.0f; S[1] = n2 * l3 - n3 * l2; S[2] = n3 * l1 - n1 * l3; S[3] = n1 * l2 - n2 * l1;
        S[4] = u1 * r[FM1 * nf] + v1 * r[FM2 * nf] + w1 * r[FM3 * nf]; break; }
    default: { float n1 = r[FN1 * nf], n2 = r[FN2 * nf], n3 = r[FN3 * nf];
        float s24 = u1 - c1 * n1, s34 = v1 - c1 * n2, s44 = w1 - c1 * n3;
        float s54 = r[FH * nf] - c1 * r[FUN * nf];
        if (c == 3) { S[0] = 1.0f; S[1] = s24; S[2] = s34; S[3] = s44; S[4] = s54; }
        else { S[0] = 1.0f; S[1] = 2 * u1 - s24; S[2] = 2 * v1 - s34; S[3] = 2 * w1 - s44;
               S[4] = 2 * r[FH * nf] - s54; }
        break; }
    }
}

// face record from face-averaged values and the face-averaged metric row
__device__ __forceinline__ void make_record(float u1, float v1, float w1, float c1,
                                            float a1, float a2, float a3, const Params &p,
                                            float *r, int nf) {
    float ss = sqrtf(a1*a1 + a2*a2 + a3*a3);
    const float n1 = a1/ss, n2 = a2/ss, n3 = a3/ss;
    float l1, l2, l3;
    if (fabsf(n3) <= fabsf(n2)) {
        ss = sqrtf(n1*n1 + n2*n2);
        l1 = -n2/ss; l2 = n1/ss; l3 = 0.0f;
    } else {
        ss = sqrtf(n1*n1 + n3*n3);
        l1 = -n3/ss; l2 = 0.0f; l3 = n1/ss;
    }
    const float KK = ((float)p.Gamma - 1.0f)/(c1*c1);
    r[FU * nf] = u1; r[FV * nf] = v1; r[FW * nf] = w1; r[FC * nf] = c1; r[FKK * nf] = KK;
    r[FX1 * nf] = 1.0f / (2.0f * c1);
    const float v2 = (u1 * u1 + v1 * v1 + w1 * w1) * 0.5f;
    r[FV2 * nf] = v2;
    r[FUN * nf] = u1 * n1 + v1 * n2 + w1 * n3;
    r[FH * nf] = v2 + 1.0f / KK;
    r[FN1 * nf] = n1; r[FN2 * nf] = n2; r[FN3 * nf] = n3;
    r[FL1 * nf] = l1; r[FL2 * nf] = l2; r[FL3 * nf] = l3;
    r[FM1 * nf] = n2*l3 - n3*l2; r[FM2 * nf] = n3*l1 - n1*l3; r[FM3 * nf] = n1*l2 - n2*l1;
}

__device__ __forceinline__ float dot5(const float S[5], float x0, float x1, float x2, float x3, float x4) {
    return S[0]*x0 + S[1]*x1 + S[2]*x2 + S[3]*x3 + S[4]*x4;
}

// CD6 / CD8 first derivative
__device__ __forceinline__ float cd6(float sm3, float sm2, float sm1, float sp1, float sp2, float sp3) {
    return (45.0f*(sp1 - sm1) - 9.0f*(sp2 - sm2) + (sp3 - sm3)) * (1.0f / 60.0f);
}
__device__ __forceinline__ float cd8(float sm4, float sm3, float sm2, float sm1,
                                     float sp1, float sp2, float sp3, float sp4) {
    return (672.0f*(sp1 - sm1) - 168.0f*(sp2 - sm2) + 32.0f*(sp3 - sm3) - 3.0f*(sp4 - sm4)) * (1.0f / 840.0f);
}

}  // namespace ocfd
