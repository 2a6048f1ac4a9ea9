// ocfd_face.cuh -- per-face pieces shared by the inviscid sweep kernels:
// Steger-Warming split with precomputed direction constants, the
// characteristic face record and eigenvector rows, the reconstruction
// dispatch, and the one-sided boundary closures.
#pragma once
#include "ocfd_device.cuh"

namespace ocfd {

// face record kept in shared memory for characteristic schemes
constexpr int FP_N = 18;   // u1 v1 w1 c1 KK X1 v2 un H  n1 n2 n3 l1 l2 l3 m1 m2 m3
enum { FU = 0, FV, FW, FC, FKK, FX1, FV2, FUN, FH, FN1, FN2, FN3, FL1, FL2, FL3, FM1, FM2, FM3 };

template <int DIR> __device__ __forceinline__ int t_ndir(const Params &p) { return DIR == 0 ? p.nx : (DIR == 1 ? p.ny : p.nz); }
template <int DIR> __device__ __forceinline__ int t_nrow(const Params &p) { return DIR == 0 ? p.ny : p.nx; }
template <int DIR> __device__ __forceinline__ long long t_sdir(const Params &p) { return DIR == 0 ? 1LL : (DIR == 1 ? p.ys : p.zs); }
template <int DIR> __device__ __forceinline__ long long t_srow(const Params &p) { return DIR == 0 ? p.ys : 1LL; }
template <int DIR> __device__ __forceinline__ long long t_s3rd(const Params &p) { return DIR == 2 ? p.ys : p.zs; }
template <int DIR> __device__ __forceinline__ double t_h(const Params &p) { return DIR == 0 ? p.hx : (DIR == 1 ? p.hy : p.hz); }

// Steger-Warming split with the direction's |A| and A/|A| already formed
// (same operations as sw_split, src/OCFD_split.cu:92-142)
// EPS0: EPSL_SW = 0, where sqrt(E*E + 0) is exactly |E| (the square root of
// a correctly rounded square returns the operand's magnitude), so the three
// square roots reduce to fabs with the same result.
template <bool EPS0>
__device__ __forceinline__ void sw_split_pre(double tmp0, double u, double v, double w, double cc,
                                             double A1, double A2, double A3, double ss,
                                             double An1, double An2, double An3,
                                             const Params &p, double *fp, double *fm) {
    const double eps = p.epsl_sw, G = p.Gamma;
    double E1 = A1 * u + A2 * v + A3 * w;
    double E2 = E1 - cc * ss;
    double E3 = E1 + cc * ss;
    double E1P = (E1 + (EPS0 ? fabs(E1) : sqrt(E1 * E1 + eps * eps))) * 0.50;
    double E2P = (E2 + (EPS0 ? fabs(E2) : sqrt(E2 * E2 + eps * eps))) * 0.50;
    double E3P = (E3 + (EPS0 ? fabs(E3) : sqrt(E3 * E3 + eps * eps))) * 0.50;
    double E1M = E1 - E1P, E2M = E2 - E2P, E3M = E3 - E3P;
    double uc1 = u - cc * An1, uc2 = u + cc * An1;
    double vc1 = v - cc * An2, vc2 = v + cc * An2;
    double wc1 = w - cc * An3, wc2 = w + cc * An3;
    double vvc1 = (uc1 * uc1 + vc1 * vc1 + wc1 * wc1) * 0.50;
    double vvc2 = (uc2 * uc2 + vc2 * vc2 + wc2 * wc2) * 0.50;
    double vv = (G - 1.0) * (u * u + v * v + w * w);
    double W2 = p.split_C3 * cc * cc;
    const double C1 = p.split_C1;
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

// row c of the left eigenvector matrix from a face record (ptoc,
// src/OCFD_flux_charteric.cu:617-676); r[k] = record value k
__device__ __forceinline__ void L_row(const double *r, int nf, int c, double S[5]) {
    const double u1 = r[FU * nf], v1 = r[FV * nf], w1 = r[FW * nf], KK = r[FKK * nf];
    switch (c) {
    case 0: S[0] = 1.0 - KK * r[FV2 * nf]; S[1] = KK * u1; S[2] = KK * v1; S[3] = KK * w1; S[4] = -KK; break;
    case 1: {
        double l1 = r[FL1 * nf], l2 = r[FL2 * nf], l3 = r[FL3 * nf];
        S[0] = -(u1 * l1 + v1 * l2 + w1 * l3); S[1] = l1; S[2] = l2; S[3] = l3; S[4] = 0.0; break; }
    case 2: {
        double m1 = r[FM1 * nf], m2 = r[FM2 * nf], m3 = r[FM3 * nf];
        double n1 = r[FN1 * nf], n2 = r[FN2 * nf], n3 = r[FN3 * nf];
        double l1 = r[FL1 * nf], l2 = r[FL2 * nf], l3 = r[FL3 * nf];
        S[0] = -(u1 * m1 + v1 * m2 + w1 * m3);
        S[1] = n2 * l3 - n3 * l2; S[2] = n3 * l1 - n1 * l3; S[3] = n1 * l2 - n2 * l1; S[4] = 0.0; break; }
    default: {
        double X1 = r[FX1 * nf], un = r[FUN * nf], v2 = r[FV2 * nf];
        double n1 = r[FN1 * nf], n2 = r[FN2 * nf], n3 = r[FN3 * nf];
        double s41 = KK * v2 * 0.5 + X1 * un;
        double s42 = -X1 * n1 - KK * u1 * 0.5;
        double s43 = -X1 * n2 - KK * v1 * 0.5;
        double s44 = -X1 * n3 - KK * w1 * 0.5;
        if (c == 3) { S[0] = s41; S[1] = s42; S[2] = s43; S[3] = s44; S[4] = KK * 0.5; }
        else { S[0] = s41 - 2 * X1 * un; S[1] = 2 * X1 * n1 + s42; S[2] = 2 * X1 * n2 + s43;
               S[3] = 2 * X1 * n3 + s44; S[4] = KK * 0.5; }
        break; }
    }
}

// column c of the right eigenvector matrix (ctop, :678-752)
__device__ __forceinline__ void R_col(const double *r, int nf, int c, double S[5]) {
    const double u1 = r[FU * nf], v1 = r[FV * nf], w1 = r[FW * nf], c1 = r[FC * nf];
    switch (c) {
    case 0: S[0] = 1.0; S[1] = u1; S[2] = v1; S[3] = w1; S[4] = r[FV2 * nf]; break;
    case 1: { double l1 = r[FL1 * nf], l2 = r[FL2 * nf], l3 = r[FL3 * nf];
        S[0] = 0.0; S[1] = l1; S[2] = l2; S[3] = l3; S[4] = u1 * l1 + v1 * l2 + w1 * l3; break; }
    case 2: { double n1 = r[FN1 * nf], n2 = r[FN2 * nf], n3 = r[FN3 * nf];
        double l1 = r[FL1 * nf], l2 = r[FL2 * nf], l3 = r[FL3 * nf];
        S[0] = 0.0; S[1] = n2 * l3 - n3 * l2; S[2] = n3 * l1 - n1 * l3; S[3] = n1 * l2 - n2 * l1;
        S[4] = u1 * r[FM1 * nf] + v1 * r[FM2 * nf] + w1 * r[FM3 * nf]; break; }
    default: { double n1 = r[FN1 * nf], n2 = r[FN2 * nf], n3 = r[FN3 * nf];
        double s24 = u1 - c1 * n1, s34 = v1 - c1 * n2, s44 = w1 - c1 * n3;
        double s54 = r[FH * nf] - c1 * r[FUN * nf];
        if (c == 3) { S[0] = 1.0; S[1] = s24; S[2] = s34; S[3] = s44; S[4] = s54; }
        else { S[0] = 1.0; S[1] = 2 * u1 - s24; S[2] = 2 * v1 - s34; S[3] = 2 * w1 - s44;
               S[4] = 2 * r[FH * nf] - s54; }
        break; }
    }
}

// face record from face-averaged values (get_para_charteric_*, :330-418)
__device__ __forceinline__ void make_record(double u1, double v1, double w1, double c1,
                                            double a1, double a2, double a3, const Params &p,
                                            double *r, int nf) {
    CharPara cp;
    char_para(u1, v1, w1, c1, a1, a2, a3, p.Gamma, cp);
    r[FU * nf] = u1; r[FV * nf] = v1; r[FW * nf] = w1; r[FC * nf] = c1; r[FKK * nf] = cp.KK;
    r[FX1 * nf] = 1.0 / (2.0 * c1);
    double v2 = (u1 * u1 + v1 * v1 + w1 * w1) * 0.5;
    r[FV2 * nf] = v2;
    r[FUN * nf] = u1 * cp.n1 + v1 * cp.n2 + w1 * cp.n3;
    r[FH * nf] = v2 + 1.0 / cp.KK;
    r[FN1 * nf] = cp.n1; r[FN2 * nf] = cp.n2; r[FN3 * nf] = cp.n3;
    r[FL1 * nf] = cp.l1; r[FL2 * nf] = cp.l2; r[FL3 * nf] = cp.l3;
    r[FM1 * nf] = cp.m1; r[FM2 * nf] = cp.m2; r[FM3 * nf] = cp.m3;
}

// UP7 (src/OCFD_Schemes.cu:865-907) with the /420 done by div_const
__device__ __forceinline__ double up7_p_q(const double *s) {
    return div_const(-3.0*s[0] + 25.0*s[1] - 101.0*s[2] + 319.0*s[3] + 214.0*s[4]
                     - 38.0*s[5] + 4.0*s[6], 420.0, 1.0 / 420.0);
}
__device__ __forceinline__ double up7_m_q(const double *s) {
    return div_const(-3.0*s[7] + 25.0*s[6] - 101.0*s[5] + 319.0*s[4] + 214.0*s[3]
                     - 38.0*s[2] + 4.0*s[1], 420.0, 1.0 / 420.0);
}

// reconstruction of one (face, sign) of one field from v[0..7] = f(F-3..F+4)
__device__ __forceinline__ double recon_one(const Params &p, int scheme, int hflag, int sign, const double *v) {
    if (sign == 0) {
        switch (scheme) {
        case 301: return up7_p_q(v);
        case 302: return weno5_p(v);
        case 303: return weno7_p(v);
        case 304: return symbo_p(0, p.tv_lim, p.tv_max, v);
        case 305: return symbo_p(1, p.tv_lim, p.tv_max, v);
        case 306: return nnd2_p(v);
        case 307: return omp6_p(0, v);
        case 308: return omp6_p(1, v);
        case 309: return omp6_p(2, v);
        default:
            if (hflag == 1) return up7_p_q(v);
            if (hflag == 2) return weno7_p(v);
            return weno5_p(v);
        }
    }
    switch (scheme) {
    case 301: return up7_m_q(v);
    case 302: return weno5_m(v);
    case 303: return weno7_m(v);
    case 304: return symbo_m(0, p.tv_lim, p.tv_max, v);
    case 305: return symbo_m(1, p.tv_lim, p.tv_max, v);
    case 306: return nnd2_m(v);
    case 307: return omp6_m(0, v);
    case 308: return omp6_m(1, v);
    case 309: return omp6_m(2, v);
    default:
        if (hflag == 1) return up7_m_q(v);
        if (hflag == 2) return weno7_m(v);
        return weno5_m(v);
    }
}

// one-sided WENO5 candidates used by the closures, src/OCFD_bound_Scheme.cu:554-745;
// s[0..4] = f(i-2..i+2)
__device__ __forceinline__ double w5_p_left(const double *s) {
    double S0 = 0.0, tmp; const double ep = 1e-6;
    tmp = s[2] - 2.0*s[3] + s[4]; S0 += 13*tmp*tmp;
    tmp = 3.0*s[2] - 4.0*s[3] + s[4]; S0 += 3*tmp*tmp;
    double a0 = 1.0/((12.0*ep + S0)*(12.0*ep + S0));
    double q03 = (2.0*s[2] + 5.0*s[3] - s[4]);
    return a0*q03/(6.0*a0);
}
__device__ __forceinline__ double w5_m_left(const double *s) {
    double S2 = 0.0, tmp; const double ep = 1e-6;
    tmp = s[4] - 2.0*s[3] + s[2]; S2 += 13*tmp*tmp;
    tmp = s[4] - 4.0*s[3] + 3.0*s[2]; S2 += 3*tmp*tmp;
    double a2 = 1.0/((12.0*ep + S2)*(12.0*ep + S2));
    double q23 = (2.0*s[4] - 7.0*s[3] + 11.0*s[2]);
    return a2*q23/(6.0*a2);
}
__device__ __forceinline__ double w5_p_right_plus(const double *s) {
    double S1 = 0.0, S2 = 0.0, tmp; const double ep = 1e-6;
    tmp = s[1] - 2.0*s[2] + s[3]; S1 += 13*tmp*tmp;
    tmp = s[1] - s[3]; S1 += 3*tmp*tmp;
    double a1 = 6.0/((12.0*ep + S1)*(12.0*ep + S1));
    double q13 = (-s[1] + 5.0*s[2] + 2.0*s[3]);
    tmp = s[0] - 2.0*s[1] + s[2]; S2 += 13*tmp*tmp;
    tmp = s[0] - 4.0*s[1] + 3.0*s[2]; S2 += 3*tmp*tmp;
    double a2 = 1.0/((12.0*ep + S2)*(12.0*ep + S2));
    double q23 = (2.0*s[0] - 7.0*s[1] + 11.0*s[2]);
    return (a1*q13 + a2*q23)/(6.0*(a1 + a2));
}
__device__ __forceinline__ double w5_p_left_plus(const double *s) {
    double S0 = 0.0, S1 = 0.0, tmp; const double ep = 1e-6;
    tmp = s[2] - 2.0*s[3] + s[4]; S0 += 13*tmp*tmp;
    tmp = 3.0*s[2] - 4.0*s[3] + s[4]; S0 += 3*tmp*tmp;
    double a0 = 3.0/((12.0*ep + S0)*(12.0*ep + S0));
    double q03 = (2.0*s[2] + 5.0*s[3] - s[4]);
    tmp = s[1] - 2.0*s[2] + s[3]; S1 += 13*tmp*tmp;
    tmp = s[1] - s[3]; S1 += 3*tmp*tmp;
    double a1 = 6.0/((12.0*ep + S1)*(12.0*ep + S1));
    double q13 = (-s[1] + 5.0*s[2] + 2.0*s[3]);
    return (a0*q03 + a1*q13)/(6.0*(a0 + a1));
}
__device__ __forceinline__ double w5_m_right_plus(const double *s) {
    double S0 = 0.0, S1 = 0.0, tmp; const double ep = 1e-6;
    tmp = s[2] - 2.0*s[1] + s[0]; S0 += 13*tmp*tmp;
    tmp = 3.0*s[2] - 4.0*s[1] + s[0]; S0 += 3*tmp*tmp;
    double a0 = 3.0/((12.0*ep + S0)*(12.0*ep + S0));
    double q03 = (2.0*s[2] + 5.0*s[1] - s[0]);
    tmp = s[3] - 2.0*s[2] + s[1]; S1 += 13*tmp*tmp;
    tmp = s[3] - s[1]; S1 += 3*tmp*tmp;
    double a1 = 6.0/((12.0*ep + S1)*(12.0*ep + S1));
    double q13 = (-s[3] + 5.0*s[2] + 2.0*s[1]);
    return (a0*q03 + a1*q13)/(6.0*(a0 + a1));
}
__device__ __forceinline__ double w5_m_left_plus(const double *s) {
    double S1 = 0.0, S2 = 0.0, tmp; const double ep = 1e-6;
    tmp = s[3] - 2.0*s[2] + s[1]; S1 += 13*tmp*tmp;
    tmp = s[3] - s[1]; S1 += 3*tmp*tmp;
    double a1 = 6.0/((12.0*ep + S1)*(12.0*ep + S1));
    double q13 = (-s[3] + 5.0*s[2] + 2.0*s[1]);
    tmp = s[4] - 2.0*s[3] + s[2]; S2 += 13*tmp*tmp;
    tmp = s[4] - 4.0*s[3] + 3.0*s[2]; S2 += 3*tmp*tmp;
    double a2 = 1.0/((12.0*ep + S2)*(12.0*ep + S2));
    double q23 = (2.0*s[4] - 7.0*s[3] + 11.0*s[2]);
    return (a1*q13 + a2*q23)/(6.0*(a1 + a2));
}

// Closure of face F+1/2 of a line of n cells, v[t] = f(F-3+t); returns true
// when it replaces the interior scheme (OCFD_bound_scheme_kernel_p / _m with
// boundp1/boundp2/boundm1/boundm2, :748-944).  KA, KB: stencil extents
// (-ia1, ib1) of the reference kernel of this sign.
__device__ __forceinline__ bool closure(int sign, bool lo, bool hi, int KA, int KB, int F, int n,
                                        const double *v, double &out) {
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
                if (t == -1) out = v[3] + 0.5 * minmod2(v[3] - v[2], v[3] - v[2]);
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
            else if (t == -2) out = v[4] - 0.5 * minmod2(v[4] - v[3], v[4] - v[3]);
            else if (t == -3) out = w5_m_right_plus(v + 2);
            else out = weno5_m(v);
            return true;
        }
    }
    return false;
}

// stencil extents of the reference kernels per scheme and sign (P: -ia1, ib1)
__device__ __forceinline__ void extents(int scheme, bool chart, int sign, int &KA, int &KB) {
    if (chart) { KA = sign ? 4 : 3; KB = sign ? 3 : 4; return; }
    switch (scheme) {
    case 302: case 306: KA = 2; KB = 2; break;
    case 303: KA = 3; KB = 3; break;
    default: KA = sign ? 4 : 3; KB = sign ? 3 : 4; break;
    }
}


}  // namespace ocfd
