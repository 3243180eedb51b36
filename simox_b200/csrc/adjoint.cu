// adjoint.cu -- parameter gradients of the energy and of a force-matching
// loss (no counterpart in the reference, whose parameters are fixed).
//
// Model (all FP64, exact list of the reference cells):
//   * EAM: for the spline metal M the density it contributes f(r), its pair
//     phi_MM(r) and its embedding F_M(rho) are uniform cubic B-splines; every
//     other EAM term keeps the analytic forms of eam.f90 (Zhou terms) and the
//     oxygen embedding of force.f90:316-344;
//   * charges q* minimise U (the CTIP_SOLVER functional, ctip.f90:307-333);
//   * forces: FORCE (force.f90:81-140 as written) + PME at q*.
// Energy E = Epair + Egroup + U(q*).  Because q* minimises U under the fixed
// total charge, dE/dtheta = dE/dtheta at fixed q (envelope theorem).
// Loss L = sum_i |F_i - T_i|^2, w = dL/dF = 2 (F - T).  With
// S(theta, q) = sum_i w_i . F_i:
//   dL/dtheta = dS/dtheta|_q - lambda . dG/dtheta,
//   (P H P) lambda = P dS/dq,
// G = grad_q U, H its Hessian (the CTIP matvec plus 2w on atoms outside their
// charge bounds), P the projection onto zero total charge: one FP64 adjoint CG.
#include "simox_internal.cuh"

#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstring>
#include <thread>
#include <vector>

namespace sx {
namespace {

constexpr int NS = SIMOX_SPLINE_N;
constexpr int AT = 128;          // threads per CTA of the pair passes (one warp per atom)
constexpr double kWpen = SX_WPEN;

struct SplineDev {
    double r0, ihr, p0, ihp;
    double phi[NS], dens[NS], emb[NS];
    int metal;                   // 0-based species index
};

struct AdjParams {
    double3 box, ibox;
    double a, kc;
    int cap, n;
    double OF[5][4], Ore[5], Ormax[5];   // oxygen embedding pieces (force.f90:316-344)
};

// Uniform cubic B-spline basis at t (knot units): interval i (clamped to the
// 61 interior intervals), values b, first and second derivatives in t.
__device__ __forceinline__ int bsp(double t, double b[4], double db[4], double d2b[4]) {
    int i = (int)floor(t);
    i = i < 0 ? 0 : (i > NS - 4 ? NS - 4 : i);
    const double u = t - i, v = 1.0 - u, u2 = u * u, u3 = u2 * u;
    b[0] = v * v * v / 6.0;
    b[1] = (3.0 * u3 - 6.0 * u2 + 4.0) / 6.0;
    b[2] = (-3.0 * u3 + 3.0 * u2 + 3.0 * u + 1.0) / 6.0;
    b[3] = u3 / 6.0;
    db[0] = -0.5 * v * v;
    db[1] = 1.5 * u2 - 2.0 * u;
    db[2] = -1.5 * u2 + u + 0.5;
    db[3] = 0.5 * u2;
    d2b[0] = v;
    d2b[1] = 3.0 * u - 2.0;
    d2b[2] = -3.0 * u + 1.0;
    d2b[3] = u;
    return i;
}

__device__ __forceinline__ double spl(const double* c, double t, double ih, double& d1, double& d2) {
    double b[4], db[4], d2b[4];
    const int i = bsp(t, b, db, d2b);
    double s = 0.0, s1 = 0.0, s2 = 0.0;
#pragma unroll
    for (int m = 0; m < 4; m++) {
        s += c[i + m] * b[m];
        s1 += c[i + m] * db[m];
        s2 += c[i + m] * d2b[m];
    }
    d1 = s1 * ih;
    d2 = s2 * ih * ih;
    return s;
}

// Zhou term g = exp(-c (r/re - 1)) / (1 + (r/re - lam)^20) and dg/dr (eam.f90:16-23)
__device__ __forceinline__ void zhou_d(double r, double ire, double c, double lam, double& g, double& dg) {
    const double rr = r * ire, t = rr - lam;
    const double t2 = t * t, t4 = t2 * t2, t8 = t4 * t4, t16 = t8 * t8, t19 = t16 * t2 * t, t20 = t19 * t;
    const double u = 1.0 / (1.0 + t20);
    g = exp(-c * (rr - 1.0)) * u;
    dg = g * ire * (-c - 20.0 * t19 * u);
}

// density that partner Y (species sY) contributes at X, and its r-derivative
__device__ __forceinline__ void dens_at_x(const SplineDev& S, const PairTab<double>& T, int sY, double r, double& f,
                                          double& df) {
    if (sY == S.metal) {
        double d2;
        f = spl(S.dens, (r - S.r0) * S.ihr, S.ihr, df, d2);
    } else {
        double g, dg;
        zhou_d(r, T.d_inv_re, T.d_c, T.d_lam, g, dg);
        f = T.d_fe * g;
        df = T.d_fe * dg;
    }
}
// density that X contributes at Y
__device__ __forceinline__ void dens_at_y(const SplineDev& S, const PairTab<double>& T, int sX, double r, double& f,
                                          double& df) {
    if (sX == S.metal) {
        double d2;
        f = spl(S.dens, (r - S.r0) * S.ihr, S.ihr, df, d2);
    } else {
        double g, dg;
        zhou_d(r, T.e_inv_re, T.e_c, T.e_lam, g, dg);
        f = T.e_fe * g;
        df = T.e_fe * dg;
    }
}
__device__ __forceinline__ void pair_phi(const SplineDev& S, const PairTab<double>& T, int sX, int sY, double r,
                                         double& p, double& dp) {
    if (sX == S.metal && sY == S.metal) {
        double d2;
        p = spl(S.phi, (r - S.r0) * S.ihr, S.ihr, dp, d2);
    } else {
        double gA, dgA, gB, dgB;
        zhou_d(r, T.p_inv_re, T.p_alpha, T.p_kappa, gA, dgA);
        zhou_d(r, T.p_inv_re, T.p_beta, T.p_lambda, gB, dgB);
        p = T.p_A * gA - T.p_B * gB;
        dp = T.p_A * dgA - T.p_B * dgB;
    }
}
// F, F', F'' of species s at rho; 1 if s has no form in this model
__device__ __forceinline__ int embed2(const SplineDev& S, const AdjParams& P, int s, double rho, double& F, double& dF,
                                      double& d2F) {
    if (s == S.metal) {
        F = spl(S.emb, (rho - S.p0) * S.ihp, S.ihp, dF, d2F);
        return 0;
    }
    if (s == 3) {   // oxygen: five cubic pieces in rho/re - 1 (force.f90:316-344)
        const int b = rho < P.Ormax[0] ? 0 : rho < P.Ormax[1] ? 1 : rho < P.Ormax[2] ? 2 : rho < P.Ormax[3] ? 3 : 4;
        const double* cf = P.OF[b];
        const double rr = P.Ore[b], t = rho / rr - 1.0;
        F = cf[0] + cf[1] * t + cf[2] * (t * t) + cf[3] * (t * t * t);
        dF = (cf[1] + cf[2] * 2.0 * t + cf[3] * 3.0 * (t * t)) / rr;
        d2F = (2.0 * cf[2] + 6.0 * cf[3] * t) / (rr * rr);
        return 0;
    }
    F = dF = d2F = 0.0;
    return 1;
}

__device__ __forceinline__ void sep(const double4& a, const double4& b, const AdjParams& P, double& dx, double& dy,
                                    double& dz) {
    dx = a.x - b.x;
    dy = a.y - b.y;
    dz = a.z - b.z;
    dx -= P.box.x * rint(dx * P.ibox.x);
    dy -= P.box.y * rint(dy * P.ibox.y);
    dz -= P.box.z * rint(dz * P.ibox.z);
}

// Ewald real-space + CTIP pair scalar (f/r on X, force.f90:94-98, 101-140 as
// written) and its derivatives by q_X, Z_X and Z_Y
struct EsPair {
    double fs, dq_a, dZx, dZy;
};
__device__ __forceinline__ EsPair es_pair(const PairTab<double>& T, double r, double qa, double qb, double a,
                                          double kc) {
    const double ir = 1.0 / r, ir2 = ir * ir;
    const double erfcv = erfc(a * r), ea = exp(-a * a * r * r);
    const double ew = (2.0 * a / SX_SQRTPI * r * ea + erfcv) * ir2 * ir;
    const double eX = exp(-2.0 * T.xi_x * r), eY = exp(-2.0 * T.xi_y * r);
    const double djfi = eX * (2.0 * T.xi_x * T.xi_x + (1.0 + 2.0 * T.xi_x * r) * ir2);
    const double difj = eY * (2.0 * T.xi_y * T.xi_y + (1.0 + 2.0 * T.xi_y * r) * ir2);
    const double QX = T.Qx[0] + r * (T.Qx[1] + r * T.Qx[2]) + ir * (T.Qx[3] + ir * T.Qx[4]);
    const double QY = T.Qy[0] + ir * (T.Qy[3] + ir * T.Qy[4]);
    const double dfifj = eX * QX + eY * QY;
    const double ZX = T.Z_x, ZY = T.Z_y;
    EsPair o;
    o.fs = kc * qa * qb * ew + kc * ((qa * ZY + qb * ZX - qa * qb) * dfifj - qa * ZY * djfi - qb * ZX * difj) * ir;
    o.dq_a = kc * qb * ew + kc * ((ZY - qb) * dfifj - ZY * djfi) * ir;
    o.dZx = kc * (qb * dfifj - qb * difj) * ir;
    o.dZy = kc * (qa * dfifj - qa * djfi) * ir;
    return o;
}

// asym_XY of CTIP_SOLVER (ctip.f90:86-106): kc (afb_X - fifj)
__device__ __forceinline__ double asym_pair(const PairTab<double>& T, double r, double kc) {
    const double ir = 1.0 / r;
    const double eX = exp(-2.0 * T.xi_x * r), eY = exp(-2.0 * T.xi_y * r);
    const double num = eX * (T.Sx[0] + r * (T.Sx[1] + r * (T.Sx[2] + r * T.Sx[3]))) + eY * (T.Sy[0] + r * T.Sy[1]);
    const double fifj = -num * ir;
    const double afbX = -eX * (T.xi_x + ir);
    return kc * (afbX - fifj);
}

__device__ __forceinline__ int slot(int k, int cap, int nm) { return k < nm ? k : cap - 1 - (k - nm); }

// pass 1: rho, F, F', F'' per atom; Egroup
__global__ void __launch_bounds__(AT)
    adj_density_kernel(AdjParams P, const SplineDev* __restrict__ S, const PairTab<double>* __restrict__ tab,
                       const double4* __restrict__ xq, const int* __restrict__ ts, const int2* __restrict__ nn,
                       const unsigned* __restrict__ nbr, double* __restrict__ rho_s, double* __restrict__ dF,
                       double* __restrict__ d2F, double* __restrict__ acc, int* __restrict__ status) {
    __shared__ double red[AT / 32];
    const SplineDev& Sp = *S;
    const int lane = threadIdx.x & 31, wpb = blockDim.x >> 5;
    double eg = 0.0;
    int bad = 0;
    for (int X = blockIdx.x * wpb + (threadIdx.x >> 5); X < P.n; X += gridDim.x * wpb) {
        const double4 xa = xq[X];
        const int sX = ts[X];
        const int2 m = nn[X];
        const unsigned* row = nbr + (size_t)X * P.cap;
        double rho = 0.0;
        for (int k = lane; k < m.x + m.y; k += 32) {
            const int Y = (int)(row[slot(k, P.cap, m.x)] & kIdxMask);
            const int sY = ts[Y];
            double dx, dy, dz;
            sep(xa, xq[Y], P, dx, dy, dz);
            const double r = sqrt(dx * dx + dy * dy + dz * dz);
            double f, df;
            dens_at_x(Sp, tab[sX * kSpecies + sY], sY, r, f, df);
            rho += f;
        }
        rho = warp_sum(rho);
        if (lane == 0) {
            double F, d1, d2;
            if (embed2(Sp, P, sX, rho, F, d1, d2)) bad |= ST_UNSUPPORTED;
            rho_s[X] = rho;
            dF[X] = d1;
            d2F[X] = d2;
            eg += F;
        }
    }
    if (bad) atomicOr(status, bad);
    block_add<AT>(eg, acc, A_EGROUP, red);
}

// pass 2: forces (EAM + Ewald real space + CTIP) into f (original order), Epair
__global__ void __launch_bounds__(AT)
    adj_force_kernel(AdjParams P, const SplineDev* __restrict__ S, const PairTab<double>* __restrict__ tab,
                     const double4* __restrict__ xq, const int* __restrict__ ts, const int2* __restrict__ nn,
                     const unsigned* __restrict__ nbr, const double* __restrict__ dF, const int* __restrict__ sorted,
                     double* __restrict__ f, double* __restrict__ acc) {
    __shared__ double red[AT / 32];
    const SplineDev& Sp = *S;
    const int lane = threadIdx.x & 31, wpb = blockDim.x >> 5;
    double ep = 0.0;
    for (int X = blockIdx.x * wpb + (threadIdx.x >> 5); X < P.n; X += gridDim.x * wpb) {
        const double4 xa = xq[X];
        const int sX = ts[X];
        const double dFX = dF[X];
        const int2 m = nn[X];
        const unsigned* row = nbr + (size_t)X * P.cap;
        double fx = 0.0, fy = 0.0, fz = 0.0;
        for (int k = lane; k < m.x + m.y; k += 32) {
            const int Y = (int)(row[slot(k, P.cap, m.x)] & kIdxMask);
            const int sY = ts[Y];
            const double4 xb = xq[Y];
            double dx, dy, dz;
            sep(xa, xb, P, dx, dy, dz);
            const double r = sqrt(dx * dx + dy * dy + dz * dz);
            const PairTab<double>& T = tab[sX * kSpecies + sY];
            double p, dp, fa, dfa, fb, dfb;
            pair_phi(Sp, T, sX, sY, r, p, dp);
            dens_at_x(Sp, T, sY, r, fa, dfa);
            dens_at_y(Sp, T, sX, r, fb, dfb);
            const double fs = -(dp + dFX * dfa + dF[Y] * dfb) / r + es_pair(T, r, xa.w, xb.w, P.a, P.kc).fs;
            fx += fs * dx;
            fy += fs * dy;
            fz += fs * dz;
            ep += 0.5 * p;
        }
        fx = warp_sum(fx);
        fy = warp_sum(fy);
        fz = warp_sum(fz);
        if (lane == 0) {
            const int o = sorted[X];
            f[3 * o] = fx;
            f[3 * o + 1] = fy;
            f[3 * o + 2] = fz;
        }
    }
    block_add<AT>(ep, acc, A_EPAIR, red);
}

// ---------------------------------------------------------------------------
// FP32 forward (simox_adjoint_forward_precision(ctx, SIMOX_MIXED)): the pair
// terms of the two forward passes in FP32 -- each separation formed in FP64
// and its length rounded once, the spline, Zhou, erfc and Slater terms in FP32
// (CUDA's single-precision expf and erfcf) -- with FP64 sums per atom.  The
// charge solve, PME, the embedding and every adjoint and gradient kernel stay
// FP64.

__device__ __forceinline__ int bsp_f(float t, float b[4], float db[4]) {
    int i = (int)floorf(t);
    i = i < 0 ? 0 : (i > NS - 4 ? NS - 4 : i);
    const float u = t - (float)i, v = 1.f - u, u2 = u * u, u3 = u2 * u;
    b[0] = v * v * v * (1.f / 6.f);
    b[1] = (3.f * u3 - 6.f * u2 + 4.f) * (1.f / 6.f);
    b[2] = (-3.f * u3 + 3.f * u2 + 3.f * u + 1.f) * (1.f / 6.f);
    b[3] = u3 * (1.f / 6.f);
    db[0] = -0.5f * v * v;
    db[1] = 1.5f * u2 - 2.f * u;
    db[2] = -1.5f * u2 + u + 0.5f;
    db[3] = 0.5f * u2;
    return i;
}

__device__ __forceinline__ float spl_f(const double* c, float t, float ih, float& d1) {
    float b[4], db[4];
    const int i = bsp_f(t, b, db);
    float sv = 0.f, s1 = 0.f;
#pragma unroll
    for (int m = 0; m < 4; m++) {
        const float cm = (float)c[i + m];
        sv = fmaf(cm, b[m], sv);
        s1 = fmaf(cm, db[m], s1);
    }
    d1 = s1 * ih;
    return sv;
}

__device__ __forceinline__ void zhou_f(float r, float ire, float c, float lam, float& g, float& dg) {
    const float rr = r * ire, t = rr - lam;
    const float t2 = t * t, t4 = t2 * t2, t8 = t4 * t4, t16 = t8 * t8, t19 = t16 * t2 * t, t20 = t19 * t;
    const float u = 1.f / (1.f + t20);
    g = expf(-c * (rr - 1.f)) * u;
    dg = g * ire * (-c - 20.f * t19 * u);
}

__device__ __forceinline__ void dens_f(const SplineDev& S, bool spline, float fe, float ire, float c, float lam, float r,
                                       float& f, float& df) {
    if (spline) {
        f = spl_f(S.dens, (r - (float)S.r0) * (float)S.ihr, (float)S.ihr, df);
    } else {
        float g, dg;
        zhou_f(r, ire, c, lam, g, dg);
        f = fe * g;
        df = fe * dg;
    }
}

__device__ __forceinline__ void pair_phi_f(const SplineDev& S, const PairTab<double>& T, int sX, int sY, float r,
                                           float& p, float& dp) {
    if (sX == S.metal && sY == S.metal) {
        p = spl_f(S.phi, (r - (float)S.r0) * (float)S.ihr, (float)S.ihr, dp);
    } else {
        float gA, dgA, gB, dgB;
        zhou_f(r, (float)T.p_inv_re, (float)T.p_alpha, (float)T.p_kappa, gA, dgA);
        zhou_f(r, (float)T.p_inv_re, (float)T.p_beta, (float)T.p_lambda, gB, dgB);
        p = (float)T.p_A * gA - (float)T.p_B * gB;
        dp = (float)T.p_A * dgA - (float)T.p_B * dgB;
    }
}

// the Ewald real-space + CTIP force scalar of es_pair in FP32
__device__ __forceinline__ float es_fs_f(const PairTab<double>& T, float r, float qa, float qb, float a, float kc) {
    const float ir = 1.f / r, ir2 = ir * ir;
    const float erfcv = erfcf(a * r), ea = expf(-a * a * r * r);
    const float ew = (2.f * a / (float)SX_SQRTPI * r * ea + erfcv) * ir2 * ir;
    const float xx = (float)T.xi_x, xy = (float)T.xi_y;
    const float eX = expf(-2.f * xx * r), eY = expf(-2.f * xy * r);
    const float djfi = eX * (2.f * xx * xx + (1.f + 2.f * xx * r) * ir2);
    const float difj = eY * (2.f * xy * xy + (1.f + 2.f * xy * r) * ir2);
    const float QX = (float)T.Qx[0] + r * ((float)T.Qx[1] + r * (float)T.Qx[2]) + ir * ((float)T.Qx[3] + ir * (float)T.Qx[4]);
    const float QY = (float)T.Qy[0] + ir * ((float)T.Qy[3] + ir * (float)T.Qy[4]);
    const float dfifj = eX * QX + eY * QY;
    const float ZX = (float)T.Z_x, ZY = (float)T.Z_y;
    return kc * qa * qb * ew + kc * ((qa * ZY + qb * ZX - qa * qb) * dfifj - qa * ZY * djfi - qb * ZX * difj) * ir;
}

// pass 1 with FP32 pair terms: rho (FP64 sum), F, F', F'' (FP64), Egroup
__global__ void __launch_bounds__(AT)
    adj_density_f_kernel(AdjParams P, const SplineDev* __restrict__ S, const PairTab<double>* __restrict__ tab,
                         const double4* __restrict__ xq, const int* __restrict__ ts, const int2* __restrict__ nn,
                         const unsigned* __restrict__ nbr, double* __restrict__ rho_s, double* __restrict__ dF,
                         double* __restrict__ d2F, double* __restrict__ acc, int* __restrict__ status) {
    __shared__ double red[AT / 32];
    const SplineDev& Sp = *S;
    const int lane = threadIdx.x & 31, wpb = blockDim.x >> 5;
    double eg = 0.0;
    int bad = 0;
    for (int X = blockIdx.x * wpb + (threadIdx.x >> 5); X < P.n; X += gridDim.x * wpb) {
        const double4 xa = xq[X];
        const int sX = ts[X];
        const int2 m = nn[X];
        const unsigned* row = nbr + (size_t)X * P.cap;
        double rho = 0.0;
        for (int k = lane; k < m.x + m.y; k += 32) {
            const int Y = (int)(row[slot(k, P.cap, m.x)] & kIdxMask);
            const int sY = ts[Y];
            double dx, dy, dz;
            sep(xa, xq[Y], P, dx, dy, dz);
            const float r = (float)sqrt(dx * dx + dy * dy + dz * dz);
            const PairTab<double>& T = tab[sX * kSpecies + sY];
            float f, df;
            dens_f(Sp, sY == Sp.metal, (float)T.d_fe, (float)T.d_inv_re, (float)T.d_c, (float)T.d_lam, r, f, df);
            rho += (double)f;
        }
        rho = warp_sum(rho);
        if (lane == 0) {
            double F, d1, d2;
            if (embed2(Sp, P, sX, rho, F, d1, d2)) bad |= ST_UNSUPPORTED;
            rho_s[X] = rho;
            dF[X] = d1;
            d2F[X] = d2;
            eg += F;
        }
    }
    if (bad) atomicOr(status, bad);
    block_add<AT>(eg, acc, A_EGROUP, red);
}

// pass 2 with FP32 pair terms: forces (FP64 sums) into f (original order), Epair
__global__ void __launch_bounds__(AT)
    adj_force_f_kernel(AdjParams P, const SplineDev* __restrict__ S, const PairTab<double>* __restrict__ tab,
                       const double4* __restrict__ xq, const int* __restrict__ ts, const int2* __restrict__ nn,
                       const unsigned* __restrict__ nbr, const double* __restrict__ dF, const int* __restrict__ sorted,
                       double* __restrict__ f, double* __restrict__ acc) {
    __shared__ double red[AT / 32];
    const SplineDev& Sp = *S;
    const int lane = threadIdx.x & 31, wpb = blockDim.x >> 5;
    const float a = (float)P.a, kc = (float)P.kc;
    double ep = 0.0;
    for (int X = blockIdx.x * wpb + (threadIdx.x >> 5); X < P.n; X += gridDim.x * wpb) {
        const double4 xa = xq[X];
        const int sX = ts[X];
        const float dFX = (float)dF[X];
        const int2 m = nn[X];
        const unsigned* row = nbr + (size_t)X * P.cap;
        double fx = 0.0, fy = 0.0, fz = 0.0;
        for (int k = lane; k < m.x + m.y; k += 32) {
            const int Y = (int)(row[slot(k, P.cap, m.x)] & kIdxMask);
            const int sY = ts[Y];
            const double4 xb = xq[Y];
            double dx, dy, dz;
            sep(xa, xb, P, dx, dy, dz);
            const float r = (float)sqrt(dx * dx + dy * dy + dz * dz);
            const PairTab<double>& T = tab[sX * kSpecies + sY];
            float p, dp, fa, dfa, fb, dfb;
            pair_phi_f(Sp, T, sX, sY, r, p, dp);
            dens_f(Sp, sY == Sp.metal, (float)T.d_fe, (float)T.d_inv_re, (float)T.d_c, (float)T.d_lam, r, fa, dfa);
            dens_f(Sp, sX == Sp.metal, (float)T.e_fe, (float)T.e_inv_re, (float)T.e_c, (float)T.e_lam, r, fb, dfb);
            const float fs = -(dp + dFX * dfa + (float)dF[Y] * dfb) / r + es_fs_f(T, r, (float)xa.w, (float)xb.w, a, kc);
            fx += (double)fs * dx;
            fy += (double)fs * dy;
            fz += (double)fs * dz;
            ep += 0.5 * (double)p;
        }
        fx = warp_sum(fx);
        fy = warp_sum(fy);
        fz = warp_sum(fz);
        if (lane == 0) {
            const int o = sorted[X];
            f[3 * o] = fx;
            f[3 * o + 1] = fy;
            f[3 * o + 2] = fz;
        }
    }
    block_add<AT>(ep, acc, A_EPAIR, red);
}

// U = sum_i [c_i q_i + J'_i q_i^2/2 + pen_i(q_i)] + 1/2 sum_i q_i (sr_i + phi_i)
// and the gradient G_i = c_i + J'_i q_i + pen'_i + sr_i + phi_i (sorted order)
__global__ void adj_u_kernel(int n, const int* __restrict__ ts, const double* __restrict__ q,
                             const double* __restrict__ cc, const double* __restrict__ sr,
                             const double* __restrict__ phi, CtipSpecies S, double* __restrict__ G,
                             double* __restrict__ acc, int slot_u) {
    __shared__ double red[256 / 32];
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    double u = 0.0;
    if (i < n) {
        const int s = min(ts[i], 4);
        const double qi = q[i];
        const double lo = min(0.0, qi - S.qmin[s]), hi = max(0.0, qi - S.qmax[s]);
        u = cc[i] * qi + 0.5 * S.Jp[s] * qi * qi + kWpen * (lo * lo + hi * hi) + 0.5 * qi * (sr[i] + phi[i]);
        G[i] = cc[i] + S.Jp[s] * qi + 2.0 * kWpen * (lo + hi) + sr[i] + phi[i];
    }
    block_add<256>(u, acc, slot_u, red);
}

// out = Hv: phi(v) (already in out) + J' v + sr(v) + 2w v on atoms outside their bounds
__global__ void adj_hess_finish(int n, const int* __restrict__ ts, const double* __restrict__ q,
                                const double* __restrict__ v, const double* __restrict__ sr, CtipSpecies S,
                                double* __restrict__ out) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const int s = min(ts[i], 4);
    const double qi = q[i];
    const bool act = qi < S.qmin[s] || qi > S.qmax[s];
    out[i] += S.Jp[s] * v[i] + sr[i] + (act ? 2.0 * kWpen * v[i] : 0.0);
}

// vector helpers for the projected CG: sum reductions into red8[k]
__global__ void adj_dot(int n, const double* __restrict__ a, const double* __restrict__ b, double* __restrict__ out) {
    __shared__ double red[256 / 32];
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    double v = i < n ? (b ? a[i] * b[i] : a[i]) : 0.0;
    block_add<256>(v, out, 0, red);
}
__global__ void adj_axpy(int n, const double* __restrict__ coef, int which, double sign, const double* __restrict__ x,
                         double* __restrict__ y) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) y[i] += sign * coef[which] * x[i];
}
__global__ void adj_sub_mean(int n, const double* __restrict__ sum, double* __restrict__ y) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) y[i] -= sum[0] / (double)n;
}
// p = r + beta p, beta = rr_new / rr_old
__global__ void adj_dir(int n, const double* __restrict__ s, const double* __restrict__ r, double* __restrict__ p) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) p[i] = r[i] + (s[1] / s[0]) * p[i];
}

// Scalars of the device-side projected CG (one block of CG_SLOTS doubles).
enum CgSlot {
    CG_MEAN = 0,    // sum for the projection onto zero mean
    CG_RN = 1,      // r.r after the update
    CG_PHP = 2,     // p.Hp
    CG_RR = 3,      // r.r of the current iterate
    CG_ALPHA = 4,   // step length
    CG_THR = 5,     // stop when r.r <= CG_THR (rtol^2 r0.r0)
    CG_K = 6,       // completed iterations
    CG_STOP = 7,    // 0 running, 1 converged, 2 p.Hp <= 0 (iterate kept), 3 non-finite residual
    CG_CHUNK = 8,   // iterations of the current graph launch
    CG_BOLD = 10,   // (old, new) r.r for adj_dir
    CG_BNEW = 11,
    CG_SLOTS = 16
};

__global__ void cg_alpha_kernel(double* __restrict__ d) {
    const double php = d[CG_PHP];
    if (php > 0.0) {
        d[CG_ALPHA] = d[CG_RR] / php;
    } else {   // not positive definite along p: no update, stop
        d[CG_ALPHA] = 0.0;
        d[CG_STOP] = 2.0;
    }
}

// End of one iteration: count it, test convergence, hand beta's terms to
// adj_dir and set the WHILE condition (at most `chunk` iterations per launch).
__global__ void cg_cond_kernel(cudaGraphConditionalHandle h, double* __restrict__ d, int maxit, int chunk) {
    bool stop = d[CG_STOP] != 0.0;
    if (!stop) {
        const double k = d[CG_K] + 1.0, rn = d[CG_RN];
        d[CG_K] = k;
        d[CG_BOLD] = d[CG_RR];
        d[CG_BNEW] = rn;
        d[CG_RR] = rn;
        if (!isfinite(rn)) {
            d[CG_STOP] = 3.0;
            stop = true;
        } else if (rn <= d[CG_THR]) {
            d[CG_STOP] = 1.0;
            stop = true;
        } else if (k >= (double)maxit) {
            stop = true;
        }
    }
    const double kc = d[CG_CHUNK] + 1.0;
    d[CG_CHUNK] = kc;
    cudaGraphSetConditional(h, (stop || kc >= (double)chunk) ? 0u : 1u);
}

// loss weights: w = 2 (F - T) in sorted order, loss, mean of w
__global__ void adj_weights(int n, const int* __restrict__ sorted, const double* __restrict__ f,
                            const double* __restrict__ T, double* __restrict__ w, double* __restrict__ acc) {
    __shared__ double red[256 / 32];
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    double l = 0.0, m0 = 0.0, m1 = 0.0, m2 = 0.0;
    if (k < n) {
        const int o = sorted[k];
        const double d0 = f[3 * o] - T[3 * o], d1 = f[3 * o + 1] - T[3 * o + 1], d2 = f[3 * o + 2] - T[3 * o + 2];
        w[3 * k] = 2.0 * d0;
        w[3 * k + 1] = 2.0 * d1;
        w[3 * k + 2] = 2.0 * d2;
        l = d0 * d0 + d1 * d1 + d2 * d2;
        m0 = 2.0 * d0;
        m1 = 2.0 * d1;
        m2 = 2.0 * d2;
    }
    block_add<256>(l, acc, 0, red);
    block_add<256>(m0, acc, 1, red);
    block_add<256>(m1, acc, 2, red);
    block_add<256>(m2, acc, 3, red);
}
__global__ void adj_center(int n, const double* __restrict__ w, const double* __restrict__ acc,
                           double* __restrict__ wt) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= n) return;
    for (int d = 0; d < 3; d++) wt[3 * k + d] = w[3 * k + d] - acc[1 + d] / (double)n;
}

// Per-CTA gradient bins in shared memory, added to the global vectors once.
// Layout of g[]: phi[64] dens[64] emb[64] (then chi J Z per species).
__device__ __forceinline__ void bin4(double* b, int i, const double v[4], double s) {
#pragma unroll
    for (int m = 0; m < 4; m++) atomicAdd(b + i + m, s * v[m]);
}

// pass 3: Gamma_X = sum_Y f'_{Y->X} (w_X - w_Y).dhat and the pair part of
// u_X = dS/dq_X = sum_Y dfs/dq_X (w_X - w_Y).d
__global__ void __launch_bounds__(AT)
    adj_gamma_kernel(AdjParams P, const SplineDev* __restrict__ S, const PairTab<double>* __restrict__ tab,
                     const double4* __restrict__ xq, const int* __restrict__ ts, const int2* __restrict__ nn,
                     const unsigned* __restrict__ nbr, const double* __restrict__ w, double* __restrict__ gam,
                     double* __restrict__ u) {
    const SplineDev& Sp = *S;
    const int lane = threadIdx.x & 31, wpb = blockDim.x >> 5;
    for (int X = blockIdx.x * wpb + (threadIdx.x >> 5); X < P.n; X += gridDim.x * wpb) {
        const double4 xa = xq[X];
        const int sX = ts[X];
        const int2 m = nn[X];
        const unsigned* row = nbr + (size_t)X * P.cap;
        const double wx = w[3 * X], wy = w[3 * X + 1], wz = w[3 * X + 2];
        double g = 0.0, uq = 0.0;
        for (int k = lane; k < m.x + m.y; k += 32) {
            const int Y = (int)(row[slot(k, P.cap, m.x)] & kIdxMask);
            const int sY = ts[Y];
            const double4 xb = xq[Y];
            double dx, dy, dz;
            sep(xa, xb, P, dx, dy, dz);
            const double r = sqrt(dx * dx + dy * dy + dz * dz);
            const double wd = (wx - w[3 * Y]) * dx + (wy - w[3 * Y + 1]) * dy + (wz - w[3 * Y + 2]) * dz;
            const PairTab<double>& T = tab[sX * kSpecies + sY];
            double fa, dfa;
            dens_at_x(Sp, T, sY, r, fa, dfa);
            g += dfa * wd / r;
            uq += es_pair(T, r, xa.w, xb.w, P.a, P.kc).dq_a * wd;
        }
        g = warp_sum(g);
        uq = warp_sum(uq);
        if (lane == 0) {
            gam[X] = g;
            u[X] = uq;
        }
    }
}

// pass 4: EAM spline gradients of E and S, and dS/dZ at fixed charges
__global__ void __launch_bounds__(AT)
    adj_grad_kernel(AdjParams P, const SplineDev* __restrict__ S, const PairTab<double>* __restrict__ tab,
                    const double4* __restrict__ xq, const int* __restrict__ ts, const int2* __restrict__ nn,
                    const unsigned* __restrict__ nbr, const double* __restrict__ w, const double* __restrict__ rho_s,
                    const double* __restrict__ dF, const double* __restrict__ d2F, const double* __restrict__ gam,
                    double* __restrict__ gE, double* __restrict__ gL, int want_L) {
    __shared__ double bE[3 * NS], bL[3 * NS + 3 * SIMOX_NATOM];
    for (int k = threadIdx.x; k < 3 * NS; k += blockDim.x) bE[k] = 0.0;
    for (int k = threadIdx.x; k < 3 * NS + 3 * SIMOX_NATOM; k += blockDim.x) bL[k] = 0.0;
    __syncthreads();
    const SplineDev& Sp = *S;
    const int lane = threadIdx.x & 31, wpb = blockDim.x >> 5;
    for (int X = blockIdx.x * wpb + (threadIdx.x >> 5); X < P.n; X += gridDim.x * wpb) {
        const double4 xa = xq[X];
        const int sX = ts[X];
        const int2 m = nn[X];
        const unsigned* row = nbr + (size_t)X * P.cap;
        const double wx = w ? w[3 * X] : 0.0, wy = w ? w[3 * X + 1] : 0.0, wz = w ? w[3 * X + 2] : 0.0;
        const double FpX = dF[X], FppX = d2F[X], gX = gam ? gam[X] : 0.0;
        for (int k = lane; k < m.x + m.y; k += 32) {
            const int Y = (int)(row[slot(k, P.cap, m.x)] & kIdxMask);
            const int sY = ts[Y];
            const double4 xb = xq[Y];
            double dx, dy, dz;
            sep(xa, xb, P, dx, dy, dz);
            const double r = sqrt(dx * dx + dy * dy + dz * dz);
            const double wd = w ? ((wx - w[3 * Y]) * dx + (wy - w[3 * Y + 1]) * dy + (wz - w[3 * Y + 2]) * dz) : 0.0;
            const double dw = wd / r;   // (w_X - w_Y) . dhat
            if (sY == Sp.metal || sX == Sp.metal) {
                double b[4], db[4], d2b[4];
                const int i = bsp((r - Sp.r0) * Sp.ihr, b, db, d2b);
                for (int mm = 0; mm < 4; mm++) db[mm] *= Sp.ihr;
                if (sX == Sp.metal && sY == Sp.metal) {
                    bin4(bE, i, b, 0.5);                       // dE/dphi_k: each pair once
                    if (want_L) bin4(bL, i, db, -0.5 * dw);    // dS/dphi_k
                }
                if (sY == Sp.metal) {                           // Y's density at X
                    bin4(bE + NS, i, b, FpX);
                    if (want_L) {
                        bin4(bL + NS, i, db, -FpX * dw);
                        bin4(bL + NS, i, b, -FppX * gX);
                    }
                }
            }
            if (want_L) {   // dS/dZ at fixed charges (each ordered pair half)
                const EsPair e = es_pair(tab[sX * kSpecies + sY], r, xa.w, xb.w, P.a, P.kc);
                atomicAdd(&bL[3 * NS + 3 * min(sX, 4) + 2], 0.5 * e.dZx * wd);
                atomicAdd(&bL[3 * NS + 3 * min(sY, 4) + 2], 0.5 * e.dZy * wd);
            }
        }
        if (lane == 0 && sX == Sp.metal) {
            double b[4], db[4], d2b[4];
            const int i = bsp((rho_s[X] - Sp.p0) * Sp.ihp, b, db, d2b);
            for (int mm = 0; mm < 4; mm++) db[mm] *= Sp.ihp;
            bin4(bE + 2 * NS, i, b, 1.0);                       // dE/demb_k
            if (want_L) bin4(bL + 2 * NS, i, db, -gX);          // dS/demb_k
        }
    }
    __syncthreads();
    for (int k = threadIdx.x; k < 3 * NS; k += blockDim.x)
        if (bE[k] != 0.0) atomicAdd(gE + k, bE[k]);
    if (want_L)
        for (int k = threadIdx.x; k < 3 * NS + 3 * SIMOX_NATOM; k += blockDim.x)
            if (bL[k] != 0.0) atomicAdd(gL + k, bL[k]);
}

// pass 5: CTIP parameter gradients.  dE: chi -> q, J -> q^2/2, Z_s -> q_X
// sum_{Y in s} asym_XY.  dL (indirect, lambda of the adjoint solve): chi ->
// -lambda, J -> -lambda q, Z_s -> -lambda_X sum_{Y in s} asym_XY.
__global__ void __launch_bounds__(AT)
    adj_ctip_grad_kernel(AdjParams P, const PairTab<double>* __restrict__ tab, const double4* __restrict__ xq,
                         const int* __restrict__ ts, const int2* __restrict__ nn, const unsigned* __restrict__ nbr,
                         const double* __restrict__ q, const double* __restrict__ lam, double* __restrict__ gE,
                         double* __restrict__ gL) {
    __shared__ double bE[3 * SIMOX_NATOM], bL[3 * SIMOX_NATOM];
    for (int k = threadIdx.x; k < 3 * SIMOX_NATOM; k += blockDim.x) bE[k] = bL[k] = 0.0;
    __syncthreads();
    const int lane = threadIdx.x & 31, wpb = blockDim.x >> 5;
    for (int X = blockIdx.x * wpb + (threadIdx.x >> 5); X < P.n; X += gridDim.x * wpb) {
        const double4 xa = xq[X];
        const int sX = min(ts[X], 4);
        const int2 m = nn[X];
        const unsigned* row = nbr + (size_t)X * P.cap;
        const double qX = q[X], lX = lam ? lam[X] : 0.0;
        for (int k = lane; k < m.x + m.y; k += 32) {
            const int Y = (int)(row[slot(k, P.cap, m.x)] & kIdxMask);
            const int sY = min(ts[Y], 4);
            double dx, dy, dz;
            sep(xa, xq[Y], P, dx, dy, dz);
            const double r = sqrt(dx * dx + dy * dy + dz * dz);
            const double as = asym_pair(tab[sX * kSpecies + min(sY, kSpecies - 1)], r, P.kc);
            atomicAdd(&bE[3 * sY + 2], qX * as);
            if (lam) atomicAdd(&bL[3 * sY + 2], -lX * as);
        }
        if (lane == 0) {
            atomicAdd(&bE[3 * sX], qX);
            atomicAdd(&bE[3 * sX + 1], 0.5 * qX * qX);
            if (lam) {
                atomicAdd(&bL[3 * sX], -lX);
                atomicAdd(&bL[3 * sX + 1], -lX * qX);
            }
        }
    }
    __syncthreads();
    for (int k = threadIdx.x; k < 3 * SIMOX_NATOM; k += blockDim.x) {
        if (bE[k] != 0.0) atomicAdd(gE + 3 * NS + k, bE[k]);
        if (lam && bL[k] != 0.0) atomicAdd(gL + 3 * NS + k, bL[k]);
    }
}

// Derivatives of one pair table entry's CTIP coefficients with respect to the
// X exponent field xi_x ([0]) and the Y field xi_y ([1]).  For X == Y the
// coefficients' whole dependence on the species' xi sits in [0].
struct XiTab {
    double dSx[2][4], dSy[2][4], dQx[2][5], dQy[2][5];
};

// pass 6: xi (zeta) gradients.  Per ordered pair (X, Y) of X's row, with
// d = d/dxi_x (credited to X's species) and d/dxi_y (to Y's):
//   dE += q_X Z_Y d asym_XY + 1/2 q_X q_Y d sym_XY          (U at fixed q)
//   dL += -lambda_X (Z_Y d asym_XY + q_Y d sym_XY)           (through G)
//       + 1/2 d fs_XY (w_X - w_Y) . d_XY                     (forces, as written)
// asym and sym are CTIP_SOLVER's (ctip.f90:86-108), fs the CTIP part of the
// pair force of force.f90:101-140.
__global__ void __launch_bounds__(AT)
    adj_xi_grad_kernel(AdjParams P, const PairTab<double>* __restrict__ tab, const XiTab* __restrict__ xit,
                       const double4* __restrict__ xq, const int* __restrict__ ts, const int2* __restrict__ nn,
                       const unsigned* __restrict__ nbr, const double* __restrict__ q,
                       const double* __restrict__ lam, const double* __restrict__ w, double* __restrict__ gE,
                       double* __restrict__ gL) {
    __shared__ PairTab<double> st[kSpecies * kSpecies];
    __shared__ XiTab sx[kSpecies * kSpecies];
    __shared__ double bE[kSpecies], bL[kSpecies];
    for (int k = threadIdx.x; k < kSpecies * kSpecies; k += blockDim.x) {
        st[k] = tab[k];
        sx[k] = xit[k];
    }
    for (int k = threadIdx.x; k < kSpecies; k += blockDim.x) bE[k] = bL[k] = 0.0;
    __syncthreads();
    const int lane = threadIdx.x & 31, wpb = blockDim.x >> 5;
    const double kc = P.kc;
    const bool want_L = lam != nullptr || w != nullptr;
    for (int X = blockIdx.x * wpb + (threadIdx.x >> 5); X < P.n; X += gridDim.x * wpb) {
        const int sX = ts[X];
        if (sX >= kSpecies) continue;
        const double4 xa = xq[X];
        const int2 m = nn[X];
        const unsigned* row = nbr + (size_t)X * P.cap;
        const double qX = q[X], lX = lam ? lam[X] : 0.0;
        const double wx = w ? w[3 * X] : 0.0, wy = w ? w[3 * X + 1] : 0.0, wz = w ? w[3 * X + 2] : 0.0;
        double eX_acc = 0.0, lX_acc = 0.0;                       // d/dxi_x: species sX
        double eY_acc[kSpecies] = {}, lY_acc[kSpecies] = {};    // d/dxi_y: species sY
        for (int k = lane; k < m.x + m.y; k += 32) {
            const int Y = (int)(row[slot(k, P.cap, m.x)] & kIdxMask);
            const int sY = ts[Y];
            if (sY >= kSpecies) continue;
            double dx, dy, dz;
            sep(xa, xq[Y], P, dx, dy, dz);
            const double r = sqrt(dx * dx + dy * dy + dz * dz);
            const double ir = 1.0 / r, ir2 = ir * ir;
            const PairTab<double>& T = st[sX * kSpecies + sY];
            const XiTab& D = sx[sX * kSpecies + sY];
            const double eX = exp(-2.0 * T.xi_x * r), eY = exp(-2.0 * T.xi_y * r);
            const double qY = q[Y], ZX = T.Z_x, ZY = T.Z_y;
            // CTIP_SOLVER pair: fifj_s = -(eX SX + eY SY)/r, afb_X = -eX (xi_x + 1/r)
            const double SX = T.Sx[0] + r * (T.Sx[1] + r * (T.Sx[2] + r * T.Sx[3]));
            const double SY = T.Sy[0] + r * T.Sy[1];
            double de[2], dl[2];
#pragma unroll
            for (int j = 0; j < 2; j++) {
                const double dSX = D.dSx[j][0] + r * (D.dSx[j][1] + r * (D.dSx[j][2] + r * D.dSx[j][3]));
                const double dSY = D.dSy[j][0] + r * D.dSy[j][1];
                const double dnum = eX * dSX + eY * dSY + (j == 0 ? -2.0 * r * eX * SX : -2.0 * r * eY * SY);
                const double dfifj_s = -dnum * ir;
                const double dafb = j == 0 ? eX * (2.0 * r * T.xi_x + 1.0) : 0.0;
                const double dasym = kc * (dafb - dfifj_s), dsym = kc * dfifj_s;
                de[j] = qX * ZY * dasym + 0.5 * qX * qY * dsym;
                dl[j] = lam ? -lX * (ZY * dasym + qY * dsym) : 0.0;
            }
            if (w) {   // as-written CTIP pair force scalar (es_pair) and its xi derivatives
                const double QX = T.Qx[0] + r * (T.Qx[1] + r * T.Qx[2]) + ir * (T.Qx[3] + ir * T.Qx[4]);
                const double QY = T.Qy[0] + ir * (T.Qy[3] + ir * T.Qy[4]);
                const double djfi = eX * (2.0 * T.xi_x * T.xi_x + (1.0 + 2.0 * T.xi_x * r) * ir2);
                const double difj = eY * (2.0 * T.xi_y * T.xi_y + (1.0 + 2.0 * T.xi_y * r) * ir2);
                const double wd = (wx - w[3 * Y]) * dx + (wy - w[3 * Y + 1]) * dy + (wz - w[3 * Y + 2]) * dz;
#pragma unroll
                for (int j = 0; j < 2; j++) {
                    const double dQX = D.dQx[j][0] + r * (D.dQx[j][1] + r * D.dQx[j][2]) +
                                       ir * (D.dQx[j][3] + ir * D.dQx[j][4]);
                    const double dQY = D.dQy[j][0] + ir * (D.dQy[j][3] + ir * D.dQy[j][4]);
                    const double ddfifj = eX * dQX + eY * dQY + (j == 0 ? -2.0 * r * eX * QX : -2.0 * r * eY * QY);
                    const double ddjfi = j == 0 ? -2.0 * r * djfi + eX * (4.0 * T.xi_x + 2.0 * ir) : 0.0;
                    const double ddifj = j == 1 ? -2.0 * r * difj + eY * (4.0 * T.xi_y + 2.0 * ir) : 0.0;
                    const double dfs =
                        kc * ((qX * ZY + qY * ZX - qX * qY) * ddfifj - qX * ZY * ddjfi - qY * ZX * ddifj) * ir;
                    dl[j] += 0.5 * dfs * wd;
                }
            }
            eX_acc += de[0];
            lX_acc += dl[0];
#pragma unroll
            for (int s = 0; s < kSpecies; s++)
                if (s == sY) {
                    eY_acc[s] += de[1];
                    lY_acc[s] += dl[1];
                }
        }
        eX_acc = warp_sum(eX_acc);
        lX_acc = warp_sum(lX_acc);
#pragma unroll
        for (int s = 0; s < kSpecies; s++) {
            eY_acc[s] = warp_sum(eY_acc[s]);
            lY_acc[s] = warp_sum(lY_acc[s]);
        }
        if (lane == 0) {
            atomicAdd(&bE[sX], eX_acc);
            if (want_L) atomicAdd(&bL[sX], lX_acc);
            for (int s = 0; s < kSpecies; s++) {
                atomicAdd(&bE[s], eY_acc[s]);
                if (want_L) atomicAdd(&bL[s], lY_acc[s]);
            }
        }
    }
    __syncthreads();
    for (int k = threadIdx.x; k < kSpecies; k += blockDim.x) {
        if (bE[k] != 0.0) atomicAdd(gE + 3 * NS + 3 * SIMOX_NATOM + k, bE[k]);
        if (want_L && bL[k] != 0.0) atomicAdd(gL + 3 * NS + 3 * SIMOX_NATOM + k, bL[k]);
    }
}

// charges of the sorted order from xq_s.w
__global__ void adj_load_q(int n, const double4* __restrict__ xq, double* __restrict__ out) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k < n) out[k] = xq[k].w;
}

// refined charges back into q (original order) and xq_s.w
__global__ void adj_store_q(int n, const int* __restrict__ sorted, const double* __restrict__ qs,
                            double* __restrict__ q, double4* __restrict__ xq) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= n) return;
    q[sorted[k]] = qs[k];
    xq[k].w = qs[k];
}

}  // namespace

// ---------------------------------------------------------------------------
// host side

struct AdjointState {
    SplineDev* spl = nullptr;
    SplineDev h{};
    double *d2F = nullptr, *w = nullptr, *wt = nullptr, *gam = nullptr, *u = nullptr, *lam = nullptr;
    double *r = nullptr, *p = nullptr, *Hp = nullptr, *sr = nullptr, *cc = nullptr, *G = nullptr, *tgt = nullptr;
    double *scal = nullptr, *gE = nullptr, *gL = nullptr;
    double* cg = nullptr;   // scalars of the device-side CG loop (CG_* slots)
    XiTab* xit = nullptr;   // d/dxi of the CTIP pair coefficients
    int cap = 0;
};

void adjoint_free(simox_ctx* c) {
    AdjointState* A = c->adj;
    if (!A) return;
    void* b[] = {A->spl, A->d2F, A->w, A->wt, A->gam, A->u, A->lam, A->r, A->p, A->Hp, A->sr, A->cc, A->G, A->tgt,
                 A->scal, A->gE, A->gL, A->cg, A->xit};
    for (void* x : b)
        if (x) cudaFree(x);
    delete A;
    c->adj = nullptr;
}

static int adjoint_alloc(simox_ctx* c) {
    if (c->adj && c->adj->cap >= c->cap) return SIMOX_OK;
    adjoint_free(c);
    AdjointState* A = new AdjointState;
    c->adj = A;
    const size_t N = (size_t)std::max(c->cap, 1);
    bool ok = cudaMalloc(&A->spl, sizeof(SplineDev)) == cudaSuccess;
    double** vec[] = {&A->d2F, &A->gam, &A->u, &A->lam, &A->r, &A->p, &A->Hp, &A->sr, &A->cc, &A->G};
    for (double** v : vec) ok = ok && cudaMalloc(v, sizeof(double) * N) == cudaSuccess;
    ok = ok && cudaMalloc(&A->w, sizeof(double) * 3 * N) == cudaSuccess &&
         cudaMalloc(&A->wt, sizeof(double) * 3 * N) == cudaSuccess &&
         cudaMalloc(&A->tgt, sizeof(double) * 3 * N) == cudaSuccess &&
         cudaMalloc(&A->scal, sizeof(double) * 8) == cudaSuccess &&
         cudaMalloc(&A->cg, sizeof(double) * CG_SLOTS) == cudaSuccess &&
         cudaMalloc(&A->xit, sizeof(XiTab) * kSpecies * kSpecies) == cudaSuccess &&
         cudaMalloc(&A->gE, sizeof(double) * SIMOX_NGRAD) == cudaSuccess &&
         cudaMalloc(&A->gL, sizeof(double) * SIMOX_NGRAD) == cudaSuccess;
    if (!ok) {
        adjoint_free(c);
        return SIMOX_E_NOMEM;
    }
    A->cap = c->cap;
    return SIMOX_OK;
}

// Dual number with two derivative components (forward-mode d/dxi_x, d/dxi_y).
struct Dual2 {
    double v, d0, d1;
    Dual2(double x = 0.0) : v(x), d0(0.0), d1(0.0) {}
    Dual2(double x, double a, double b) : v(x), d0(a), d1(b) {}
};
static inline Dual2 operator+(Dual2 a, Dual2 b) { return {a.v + b.v, a.d0 + b.d0, a.d1 + b.d1}; }
static inline Dual2 operator-(Dual2 a, Dual2 b) { return {a.v - b.v, a.d0 - b.d0, a.d1 - b.d1}; }
static inline Dual2 operator*(Dual2 a, Dual2 b) {
    return {a.v * b.v, a.d0 * b.v + a.v * b.d0, a.d1 * b.v + a.v * b.d1};
}
static inline Dual2 operator/(Dual2 a, Dual2 b) {
    const double q = a.v / b.v;
    return {q, (a.d0 - q * b.d0) / b.v, (a.d1 - q * b.d1) / b.v};
}

// d/dxi tables: the coefficient construction of the pair tables (fafb from
// datafmt.f90:201-220, then the force.f90 / ctip.f90 polynomials) run on dual
// numbers seeded with d xi_x = (1, 0), d xi_y = (0, 1).
static void xi_tables(const simox_potential& pot, XiTab* out) {
    for (int X = 0; X < kSpecies; X++)
        for (int Y = 0; Y < kSpecies; Y++) {
            const bool same = X == Y;
            const Dual2 xx(pot.param[X].xi, 1.0, 0.0);
            const Dual2 xy = same ? xx : Dual2(pot.param[Y].xi, 0.0, 1.0);
            Dual2 f[4], Px[5], Py[5], Qx[5], Qy[5], Sx[4], Sy[4];
            slater_fafb<Dual2>(xx, xy, same, f);
            ctip_coefs<Dual2>(xx, xy, same, f, Px, Py, Qx, Qy, Sx, Sy);
            XiTab& t = out[X * kSpecies + Y];
            for (int k = 0; k < 5; k++) {
                t.dQx[0][k] = Qx[k].d0; t.dQx[1][k] = Qx[k].d1;
                t.dQy[0][k] = Qy[k].d0; t.dQy[1][k] = Qy[k].d1;
            }
            for (int k = 0; k < 4; k++) {
                t.dSx[0][k] = Sx[k].d0; t.dSx[1][k] = Sx[k].d1;
                t.dSy[0][k] = Sy[k].d0; t.dSy[1][k] = Sy[k].d1;
            }
        }
}

static AdjParams adj_params(const simox_ctx* c) {
    AdjParams P;
    P.box = make_double3(c->box[0], c->box[1], c->box[2]);
    P.ibox = make_double3(c->inv_box[0], c->inv_box[1], c->inv_box[2]);
    P.a = c->a;
    P.kc = SX_KC;
    P.cap = c->nnb_cap;
    P.n = c->n;
    const simox_oxid& o = c->pot.oxygn;
    const double* Fb[5] = {o.F0, o.F1, o.F2, o.F3, o.F4};
    for (int b = 0; b < 5; b++) {
        for (int k = 0; k < 4; k++) P.OF[b][k] = Fb[b][k];
        P.Ore[b] = o.re[b];
        P.Ormax[b] = o.rmax[b];
    }
    return P;
}

// Hv (sorted order): c_pme phi(v) + J' v + sr(v) + 2w v on atoms outside bounds
static int hess(simox_ctx* c, const CtipSpecies& S, double c_pme, const double* v, double* out) {
    AdjointState* A = c->adj;
    int st = pme_potential(c, v, out, c_pme);
    if (st) return st;
    ctip_pair(c, v, A->sr, nullptr, S);
    const int nb = (c->n + 255) / 256;
    Launch L(c, "adjoint_hess");
    adj_hess_finish<<<nb, 256, 0, c->stream>>>(c->n, c->t_s, c->qs, v, A->sr, S, out);
    return check_launch(c);
}

static double host_scalar(simox_ctx* c, const double* d, int k = 0) {
    double h[8];
    cudaMemcpyAsync(h, d, sizeof(double) * 8, cudaMemcpyDeviceToHost, c->stream);
    cudaStreamSynchronize(c->stream);
    return h[k];
}

// y -= mean(y), the sum reduced into *sum
static void project(simox_ctx* c, double* y, double* sum) {
    const int n = c->n, nb = (n + 255) / 256;
    cudaMemsetAsync(sum, 0, sizeof(double), c->stream);
    adj_dot<<<nb, 256, 0, c->stream>>>(n, y, nullptr, sum);
    adj_sub_mean<<<nb, 256, 0, c->stream>>>(n, sum, y);
}

// Iterations per graph launch of the device-side CG loop: every launch ends
// after a bounded time and the host checks the status between launches.
constexpr int kCgIterChunk = 256;

// Projected CG iterations on the device.  One iteration (H p, projection,
// p.Hp, step, residual, direction) is the body of a CUDA graph WHILE node;
// cg_alpha_kernel and cg_cond_kernel take the decisions the host loop takes.
// Expects b = r (projected), p = r, x = 0 and r0 = r.r.  *used = false (nothing
// run) when the graph cannot be built here.
static int proj_cg_device(simox_ctx* c, const CtipSpecies& S, double c_pme, double* b, double* x, double r0,
                          double rtol, int maxit, int* k_out, double* rr_out, bool* used) {
    *used = false;
    if (c->profiling) return SIMOX_OK;
    AdjointState* A = c->adj;
    const int n = c->n, nb = (n + 255) / 256;
    const cudaStream_t s = c->stream;
    double* d = A->cg;
    cudaGraph_t outer = nullptr;
    cudaGraphExec_t exec = nullptr;
    if (cudaGraphCreate(&outer, 0) != cudaSuccess) {
        cudaGetLastError();
        return SIMOX_OK;
    }
    cudaGraphConditionalHandle h;
    cudaGraphNodeParams np{};
    cudaGraphNode_t node;
    bool ok = cudaGraphConditionalHandleCreate(&h, outer, 1u, cudaGraphCondAssignDefault) == cudaSuccess;
    if (ok) {
        np.type = cudaGraphNodeTypeConditional;
        np.conditional.handle = h;
        np.conditional.type = cudaGraphCondTypeWhile;
        np.conditional.size = 1;
        ok = cudaGraphAddNode(&node, outer, nullptr, 0, &np) == cudaSuccess;
    }
    long long per_iter = 0;
    int st = SIMOX_OK;
    if (ok) {
        cudaGraph_t body = np.conditional.phGraph_out[0];
        ok = cudaStreamBeginCaptureToGraph(s, body, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal) ==
             cudaSuccess;
        if (ok) {
            const long long l0 = c->launches;
            st = hess(c, S, c_pme, A->p, A->Hp);
            project(c, A->Hp, d + CG_MEAN);
            cudaMemsetAsync(d + CG_PHP, 0, sizeof(double), s);
            adj_dot<<<nb, 256, 0, s>>>(n, A->p, A->Hp, d + CG_PHP);
            cg_alpha_kernel<<<1, 1, 0, s>>>(d);
            adj_axpy<<<nb, 256, 0, s>>>(n, d, CG_ALPHA, 1.0, A->p, x);
            adj_axpy<<<nb, 256, 0, s>>>(n, d, CG_ALPHA, -1.0, A->Hp, b);
            cudaMemsetAsync(d + CG_RN, 0, sizeof(double), s);
            adj_dot<<<nb, 256, 0, s>>>(n, b, b, d + CG_RN);
            cg_cond_kernel<<<1, 1, 0, s>>>(h, d, maxit, kCgIterChunk);
            adj_dir<<<nb, 256, 0, s>>>(n, d + CG_BOLD, b, A->p);
            cudaGraph_t cap = nullptr;
            ok = cudaStreamEndCapture(s, &cap) == cudaSuccess && st == SIMOX_OK;
            per_iter = c->launches - l0 + 9;   // + the nine vector and scalar kernels above
            c->launches = l0;
        }
        ok = ok && cudaGraphInstantiate(&exec, outer, 0) == cudaSuccess;
    }
    cudaGetLastError();
    if (!ok) {
        if (exec) cudaGraphExecDestroy(exec);
        cudaGraphDestroy(outer);
        return st;
    }
    *used = true;
    double hd[CG_SLOTS] = {};
    hd[CG_RR] = r0;
    hd[CG_THR] = rtol * rtol * r0;
    cudaMemcpyAsync(d, hd, sizeof(hd), cudaMemcpyHostToDevice, s);
    int k = 0;
    while (true) {
        cudaMemsetAsync(d + CG_CHUNK, 0, sizeof(double), s);
        if ((st = cuda_status(cudaGraphLaunch(exec, s)))) break;
        cudaMemcpyAsync(hd, d, sizeof(hd), cudaMemcpyDeviceToHost, s);
        if ((st = cuda_status(cudaStreamSynchronize(s)))) break;
        const int k_now = (int)hd[CG_K];
        c->launches += per_iter * (long long)(k_now - k);
        k = k_now;
        if (hd[CG_STOP] != 0.0 || k >= maxit) break;
    }
    *k_out = k;
    *rr_out = hd[CG_RR];
    cudaGraphExecDestroy(exec);
    cudaGraphDestroy(outer);
    return st;
}

// projected CG: (P H P) x = P b, x orthogonal to the all-ones vector.
// x must start at zero; b is overwritten (it becomes the residual).  The
// iterations run as a device-side graph loop, or host-driven when the graph
// cannot be built (and with the per-launch profile on).
static int proj_cg(simox_ctx* c, const CtipSpecies& S, double c_pme, double* b, double* x, double rtol, int maxit,
                   int* iters, double* relres, double abs_tol = 0.0, double* norm0 = nullptr) {
    AdjointState* A = c->adj;
    const int n = c->n, nb = (n + 255) / 256;
    double* s = A->scal;
    project(c, b, s);   // r = P b (x = 0)
    cudaMemcpyAsync(A->p, b, sizeof(double) * n, cudaMemcpyDeviceToDevice, c->stream);
    cudaMemsetAsync(s, 0, sizeof(double) * 8, c->stream);
    adj_dot<<<nb, 256, 0, c->stream>>>(n, b, b, s);            // s[0] = r.r
    const double r0 = host_scalar(c, s, 0);
    if (norm0) *norm0 = std::sqrt(r0);
    double rr = r0;
    int k = 0;
    bool device_loop = false;
    if (r0 > abs_tol * abs_tol && maxit > 0) {
        int st = proj_cg_device(c, S, c_pme, b, x, r0, rtol, maxit, &k, &rr, &device_loop);
        if (st) return st;
    }
    if (r0 > abs_tol * abs_tol && !device_loop) {
        for (k = 0; k < maxit; k++) {
            int st = hess(c, S, c_pme, A->p, A->Hp);
            if (st) return st;
            project(c, A->Hp, s);
            // s[2] = p.Hp ; alpha = rr / pHp
            cudaMemsetAsync(s + 2, 0, sizeof(double), c->stream);
            adj_dot<<<nb, 256, 0, c->stream>>>(n, A->p, A->Hp, s + 2);
            const double pHp = host_scalar(c, s, 2);
            if (!(pHp > 0.0)) break;   // not positive definite along p: keep the iterate so far
            double h[2] = {rr / pHp, 0.0};
            cudaMemcpyAsync(s + 4, h, sizeof(double), cudaMemcpyHostToDevice, c->stream);
            adj_axpy<<<nb, 256, 0, c->stream>>>(n, s, 4, 1.0, A->p, x);
            adj_axpy<<<nb, 256, 0, c->stream>>>(n, s, 4, -1.0, A->Hp, b);
            cudaMemsetAsync(s + 1, 0, sizeof(double), c->stream);
            adj_dot<<<nb, 256, 0, c->stream>>>(n, b, b, s + 1);   // s[1] = new r.r
            const double rn = host_scalar(c, s, 1);
            if (rn <= rtol * rtol * r0) {
                rr = rn;
                k++;
                break;
            }
            double hs[2] = {rr, rn};
            cudaMemcpyAsync(s, hs, sizeof(double) * 2, cudaMemcpyHostToDevice, c->stream);
            adj_dir<<<nb, 256, 0, c->stream>>>(n, s, b, A->p);
            rr = rn;
        }
    }
    *iters = k;
    *relres = r0 > 0.0 ? std::sqrt(rr / r0) : 0.0;
    return check_launch(c);
}

int adjoint_eval(simox_ctx* c, const double* f_target, simox_adjoint_report* rep, double* forces, double* grad_E,
                 double* grad_L) {
    if (!c->adj || !c->spline_on) return SIMOX_E_STATE;
    if (!c->psi_valid || !c->cells_valid) return SIMOX_E_STATE;
    if (c->precision != SIMOX_FP64) return SIMOX_E_UNSUPPORTED;
    AdjointState* A = c->adj;
    simox_adjoint_report R;
    std::memset(&R, 0, sizeof(R));
    const int n = c->n, nb = (n + 255) / 256;
    const cudaStream_t s = c->stream;
    const CtipSpecies S = ctip_species(c);
    const double V = c->box[0] * c->box[1] * c->box[2];
    const double c_pme = SX_KC * (double)c->fft[0] * (double)c->fft[1] * (double)c->fft[2] / V / SX_PI;
    int st;
    // charges: the reference's CG, then Newton steps on the fixed active set.
    // The entry charges (sorted order) are kept in u, free until the loss pass.
    if ((st = ensure_list(c))) return st;
    adj_load_q<<<nb, 256, 0, s>>>(n, c->xq_s, A->u);
    simox_ctip_report cr{};
    if (!c->adj_warm && (st = ctip_solve(c, 0, &cr))) return st;
    R.n_cg = cr.n_cg;
    if (c->adj_warm) adj_load_q<<<nb, 256, 0, s>>>(n, c->xq_s, c->qs);   // the held charges, in pair order
    auto grad_u = [&](double* Uout) -> int {
        // c (chi + sum Z asym), sr = sym q, phi = c_pme phi(q); G and U
        ctip_pair(c, c->qs, A->sr, A->cc, S);
        if (int e = pme_potential(c, c->qs, A->Hp, c_pme)) return e;
        cudaMemsetAsync(A->scal, 0, sizeof(double) * 8, s);
        adj_u_kernel<<<nb, 256, 0, s>>>(n, c->t_s, c->qs, A->cc, A->sr, A->Hp, S, A->G, A->scal, 0);
        if (Uout) *Uout = host_scalar(c, A->scal, 0);
        return check_launch(c);
    };
    // ||P G|| at the current charges (G from grad_u)
    auto resid = [&]() -> double {
        cudaMemcpyAsync(A->r, A->G, sizeof(double) * n, cudaMemcpyDeviceToDevice, s);
        cudaMemsetAsync(A->scal, 0, sizeof(double) * 8, s);
        adj_dot<<<nb, 256, 0, s>>>(n, A->r, nullptr, A->scal);
        adj_sub_mean<<<nb, 256, 0, s>>>(n, A->scal, A->r);
        cudaMemsetAsync(A->scal + 1, 0, sizeof(double), s);
        adj_dot<<<nb, 256, 0, s>>>(n, A->r, A->r, A->scal + 1);
        return std::sqrt(host_scalar(c, A->scal, 1));
    };
    // Safeguarded Newton: the CTIP functional is convex only where the charge
    // penalties hold it (J' is smaller than the Coulomb coupling of an
    // alternating charge pattern), so a step is solved on the current active
    // set and accepted (halving up to 4 times) only if it lowers ||P G||.
    const double abs_tol = 1e-11 * std::sqrt((double)n);
    auto newton = [&](double& rn, int& steps) -> int {
        for (int it = 0; it < 8 && rn > abs_tol; it++) {
            cudaMemsetAsync(A->lam, 0, sizeof(double) * n, s);
            {
                double m1 = -1.0;
                cudaMemcpyAsync(A->scal + 4, &m1, sizeof(double), cudaMemcpyHostToDevice, s);
                cudaMemsetAsync(A->r, 0, sizeof(double) * n, s);
                adj_axpy<<<nb, 256, 0, s>>>(n, A->scal, 4, 1.0, A->G, A->r);   // r = -G
            }
            int its = 0;
            double rel = 0.0;
            if (int e = proj_cg(c, S, c_pme, A->r, A->lam, 1e-13, 2000, &its, &rel)) return e;
            // trial charges q + t delta; the accepted step stays in qs
            cudaMemcpyAsync(A->gam, c->qs, sizeof(double) * n, cudaMemcpyDeviceToDevice, s);   // saved q
            bool accepted = false;
            double t = 1.0;
            for (int ls = 0; ls < 5 && !accepted; ls++, t *= 0.5) {
                cudaMemcpyAsync(c->qs, A->gam, sizeof(double) * n, cudaMemcpyDeviceToDevice, s);
                cudaMemcpyAsync(A->scal + 5, &t, sizeof(double), cudaMemcpyHostToDevice, s);
                adj_axpy<<<nb, 256, 0, s>>>(n, A->scal, 5, 1.0, A->lam, c->qs);
                if (int e = grad_u(nullptr)) return e;
                const double rt = resid();
                if (rt < rn) {
                    rn = rt;
                    accepted = true;
                }
            }
            steps = it + 1;
            if (!accepted) {   // no step lowers the residual: keep the previous charges
                cudaMemcpyAsync(c->qs, A->gam, sizeof(double) * n, cudaMemcpyDeviceToDevice, s);
                if (int e = grad_u(nullptr)) return e;
                break;
            }
        }
        return SIMOX_OK;
    };
    double Uq = 0.0;
    if ((st = grad_u(nullptr))) return st;
    double rn = resid();
    int steps = 0;
    if ((st = newton(rn, steps))) return st;
    R.n_newton = steps;
    if (rn > 1e-9 * std::sqrt((double)n)) {
        // Stalled: the CG's last line search can leave the charges where the
        // functional is not convex on the current active set.  Restart the
        // refinement from the entry charges and keep the smaller residual.
        cudaMemcpyAsync(A->tgt, c->qs, sizeof(double) * n, cudaMemcpyDeviceToDevice, s);   // first result
        cudaMemcpyAsync(c->qs, A->u, sizeof(double) * n, cudaMemcpyDeviceToDevice, s);
        if ((st = grad_u(nullptr))) return st;
        double rn2 = resid();
        int steps2 = 0;
        if ((st = newton(rn2, steps2))) return st;
        R.n_newton += steps2;
        if (!(rn2 < rn)) cudaMemcpyAsync(c->qs, A->tgt, sizeof(double) * n, cudaMemcpyDeviceToDevice, s);
    }
    if ((st = grad_u(&Uq))) return st;
    {   // residual ||P G||
        cudaMemcpyAsync(A->r, A->G, sizeof(double) * n, cudaMemcpyDeviceToDevice, s);
        cudaMemsetAsync(A->scal, 0, sizeof(double) * 8, s);
        adj_dot<<<nb, 256, 0, s>>>(n, A->r, nullptr, A->scal);
        adj_sub_mean<<<nb, 256, 0, s>>>(n, A->scal, A->r);
        cudaMemsetAsync(A->scal + 1, 0, sizeof(double), s);
        adj_dot<<<nb, 256, 0, s>>>(n, A->r, A->r, A->scal + 1);
        R.residual = std::sqrt(host_scalar(c, A->scal, 1));
    }
    adj_store_q<<<nb, 256, 0, s>>>(n, c->pair_order, c->qs, c->q, c->xq_s);
    R.U = Uq;
    // forces and EAM energies of the spline model
    const AdjParams P = adj_params(c);
    const int wpb = AT / 32;
    const int g = std::max(1, std::min((n + wpb - 1) / wpb, num_sms(c) * 16));
    cudaMemsetAsync(c->acc, 0, sizeof(double) * (A_EREC + 1), s);
    if (c->adj_fwd32) {   // FP32 pair terms in the forward passes
        Launch L(c, "adjoint_forward_fp32");
        adj_density_f_kernel<<<g, AT, 0, s>>>(P, A->spl, c->tab_d, c->xq_s, c->t_s,
                                              reinterpret_cast<const int2*>(c->nn), c->nbr, c->rho_s, c->dF_s, A->d2F,
                                              c->acc, c->status);
        adj_force_f_kernel<<<g, AT, 0, s>>>(P, A->spl, c->tab_d, c->xq_s, c->t_s,
                                            reinterpret_cast<const int2*>(c->nn), c->nbr, c->dF_s, c->pair_order, c->f,
                                            c->acc);
    } else {
        {
            Launch L(c, "adjoint_density");
            adj_density_kernel<<<g, AT, 0, s>>>(P, A->spl, c->tab_d, c->xq_s, c->t_s,
                                                reinterpret_cast<const int2*>(c->nn), c->nbr, c->rho_s, c->dF_s,
                                                A->d2F, c->acc, c->status);
        }
        {
            Launch L(c, "adjoint_force");
            adj_force_kernel<<<g, AT, 0, s>>>(P, A->spl, c->tab_d, c->xq_s, c->t_s,
                                              reinterpret_cast<const int2*>(c->nn), c->nbr, c->dF_s, c->pair_order,
                                              c->f, c->acc);
        }
    }
    if ((st = pme_forces(c, true, false))) return st;
    if ((st = read_status(c))) return st;
    cudaMemcpyAsync(c->h_acc, c->acc, sizeof(double) * A_COUNT, cudaMemcpyDeviceToHost, s);
    if ((st = cuda_status(cudaStreamSynchronize(s)))) return st;
    R.E_eam = c->h_acc[A_EPAIR] + c->h_acc[A_EGROUP];
    R.E = R.E_eam + R.U;
    if (forces) {
        cudaMemcpyAsync(forces, c->f, sizeof(double) * 3 * n, cudaMemcpyDeviceToHost, s);
        if ((st = cuda_status(cudaStreamSynchronize(s)))) return st;
    }
    const bool want_L = f_target != nullptr && grad_L != nullptr;
    cudaMemsetAsync(A->gE, 0, sizeof(double) * SIMOX_NGRAD, s);
    cudaMemsetAsync(A->gL, 0, sizeof(double) * SIMOX_NGRAD, s);
    if (f_target) {
        cudaMemcpyAsync(A->tgt, f_target, sizeof(double) * 3 * n, cudaMemcpyHostToDevice, s);
        cudaMemsetAsync(A->scal, 0, sizeof(double) * 8, s);
        adj_weights<<<nb, 256, 0, s>>>(n, c->pair_order, c->f, A->tgt, A->w, A->scal);
        adj_center<<<nb, 256, 0, s>>>(n, A->w, A->scal, A->wt);
        R.loss = host_scalar(c, A->scal, 0);
    }
    if (want_L) {
        Launch L(c, "adjoint_gamma");
        adj_gamma_kernel<<<g, AT, 0, s>>>(P, A->spl, c->tab_d, c->xq_s, c->t_s, reinterpret_cast<const int2*>(c->nn),
                                          c->nbr, A->w, A->gam, A->u);
    }
    {
        Launch L(c, "adjoint_grad_eam");
        adj_grad_kernel<<<g, AT, 0, s>>>(P, A->spl, c->tab_d, c->xq_s, c->t_s, reinterpret_cast<const int2*>(c->nn),
                                         c->nbr, want_L ? A->w : nullptr, c->rho_s, c->dF_s, A->d2F,
                                         want_L ? A->gam : nullptr, A->gE, A->gL, want_L ? 1 : 0);
    }
    if (want_L) {
        // u = dS/dq: pair part (above) + PME part; then (P H P) lambda = P u
        if ((st = pme_force_charge_adjoint(c, A->wt, A->u))) return st;
        cudaMemcpyAsync(A->r, A->u, sizeof(double) * n, cudaMemcpyDeviceToDevice, s);
        cudaMemsetAsync(A->lam, 0, sizeof(double) * n, s);
        if ((st = proj_cg(c, S, c_pme, A->r, A->lam, 1e-12, 4000, &R.n_adjoint, &R.adj_residual))) return st;
    }
    {
        Launch L(c, "adjoint_grad_ctip");
        adj_ctip_grad_kernel<<<g, AT, 0, s>>>(P, c->tab_d, c->xq_s, c->t_s, reinterpret_cast<const int2*>(c->nn),
                                              c->nbr, c->qs, want_L ? A->lam : nullptr, A->gE, A->gL);
    }
    {
        XiTab hx[kSpecies * kSpecies];
        xi_tables(c->pot, hx);
        cudaMemcpyAsync(A->xit, hx, sizeof(hx), cudaMemcpyHostToDevice, s);
        Launch L(c, "adjoint_grad_xi");
        adj_xi_grad_kernel<<<g, AT, 0, s>>>(P, c->tab_d, A->xit, c->xq_s, c->t_s,
                                            reinterpret_cast<const int2*>(c->nn), c->nbr, c->qs,
                                            want_L ? A->lam : nullptr, want_L ? A->w : nullptr, A->gE, A->gL);
    }
    if ((st = check_launch(c))) return st;
    if (grad_E) cudaMemcpyAsync(grad_E, A->gE, sizeof(double) * SIMOX_NGRAD, cudaMemcpyDeviceToHost, s);
    if (grad_L) cudaMemcpyAsync(grad_L, A->gL, sizeof(double) * SIMOX_NGRAD, cudaMemcpyDeviceToHost, s);
    if ((st = cuda_status(cudaStreamSynchronize(s)))) return st;
    if (grad_L && !want_L) std::memset(grad_L, 0, sizeof(double) * SIMOX_NGRAD);
    if (rep) *rep = R;
    return SIMOX_OK;
}

int set_eam_spline(simox_ctx* c, const simox_eam_spline* sp) {
    if (!sp) {
        c->spline_on = false;
        return SIMOX_OK;
    }
    if (sp->metal < 1 || sp->metal > 3 || !(sp->r1 > sp->r0) || !(sp->rho1 > sp->rho0)) return SIMOX_E_ARG;
    if (int st = adjoint_alloc(c)) return st;
    SplineDev& h = c->adj->h;
    h.metal = sp->metal - 1;
    h.r0 = sp->r0;
    h.ihr = (double)(NS - 3) / (sp->r1 - sp->r0);
    h.p0 = sp->rho0;
    h.ihp = (double)(NS - 3) / (sp->rho1 - sp->rho0);
    std::memcpy(h.phi, sp->phi, sizeof(h.phi));
    std::memcpy(h.dens, sp->dens, sizeof(h.dens));
    std::memcpy(h.emb, sp->emb, sizeof(h.emb));
    if (cudaMemcpyAsync(c->adj->spl, &h, sizeof(SplineDev), cudaMemcpyHostToDevice, c->stream) != cudaSuccess)
        return SIMOX_E_CUDA;
    c->spline_on = true;
    // the model runs on the reference cells' exact list
    c->skin_mode = false;
    c->skin_valid = false;
    c->gathered = false;
    c->list_valid = false;
    drop_graphs(c);
    return cuda_status(cudaStreamSynchronize(c->stream));
}

}  // namespace sx

extern "C" int simox_set_eam_spline(simox_ctx* c, const simox_eam_spline* s) {
    if (!c) return SIMOX_E_ARG;
    cudaSetDevice(c->device);
    return sx::set_eam_spline(c, s);
}

extern "C" int simox_set_ctip_params(simox_ctx* c, int species, double chi, double J, double Z) {
    if (!c || species < 1 || species > SIMOX_NATOM) return SIMOX_E_ARG;
    cudaSetDevice(c->device);
    simox_potn& p = c->pot.param[species - 1];
    p.chi = chi;
    p.J = J;
    p.Z = Z;
    return sx::build_pair_tables(c);   // Z enters the pair tables
}

extern "C" int simox_set_ctip_xi(simox_ctx* c, int species, double xi) {
    if (!c || species < 1 || species > SIMOX_NATOM || !(xi > 0.0) || !std::isfinite(xi)) return SIMOX_E_ARG;
    for (int s = 0; s < SIMOX_NATOM; s++)
        if (s != species - 1 && c->pot.param[s].xi == xi) return SIMOX_E_ARG;
    cudaSetDevice(c->device);
    c->pot.param[species - 1].xi = xi;
    for (int i = 0; i < SIMOX_NATOM; i++)   // datafmt.f90:201-220 for every pair involving the species
        for (int j = 0; j < SIMOX_NATOM; j++)
            if (i == species - 1 || j == species - 1)
                sx::slater_fafb<double>(c->pot.param[i].xi, c->pot.param[j].xi, i == j, c->pot.param[i].fafb[j]);
    return sx::build_pair_tables(c);
}

// warm start of the adjoint's charge solve (see the header)
extern "C" int simox_adjoint_forward_precision(simox_ctx* c, int precision) {
    if (!c || (precision != SIMOX_FP64 && precision != SIMOX_MIXED)) return SIMOX_E_ARG;
    c->adj_fwd32 = precision == SIMOX_MIXED;
    return SIMOX_OK;
}

extern "C" int simox_adjoint_warm_start(simox_ctx* c, int on) {
    if (!c) return SIMOX_E_ARG;
    c->adj_warm = on != 0;
    return SIMOX_OK;
}

extern "C" int simox_adjoint_eval(simox_ctx* c, const double* f_target, simox_adjoint_report* rep, double* forces,
                                  double* grad_E, double* grad_L) {
    if (!c) return SIMOX_E_ARG;
    cudaSetDevice(c->device);
    return sx::adjoint_eval(c, f_target, rep, forces, grad_E, grad_L);
}

extern "C" int simox_adjoint_eval_many(simox_ctx* const* ctxs, int m, const double* const* f_target,
                                       simox_adjoint_report* reps, double* const* forces, double* const* grad_E,
                                       double* const* grad_L, int threads) {
    if (m < 0 || (m > 0 && !ctxs)) return SIMOX_E_ARG;
    for (int i = 0; i < m; i++) {
        if (!ctxs[i]) return SIMOX_E_ARG;
        for (int j = 0; j < i; j++)
            if (ctxs[j] == ctxs[i]) return SIMOX_E_ARG;   // one host thread per context at a time
    }
    if (m == 0) return SIMOX_OK;
    int nt = threads > 0 ? threads : std::min(m, 16);
    nt = std::max(1, std::min(nt, m));
    std::vector<int> st(m, SIMOX_OK);
    std::atomic<int> next{0};
    auto work = [&]() {
        for (int i = next++; i < m; i = next++) {
            simox_ctx* c = ctxs[i];
            cudaSetDevice(c->device);
            st[i] = sx::adjoint_eval(c, f_target ? f_target[i] : nullptr, reps ? reps + i : nullptr,
                                     forces ? forces[i] : nullptr, grad_E ? grad_E[i] : nullptr,
                                     grad_L ? grad_L[i] : nullptr);
        }
    };
    std::vector<std::thread> pool;
    pool.reserve(nt - 1);
    for (int t = 1; t < nt; t++) pool.emplace_back(work);
    work();
    for (std::thread& t : pool) t.join();
    for (int i = 0; i < m; i++)
        if (st[i]) return st[i];
    return SIMOX_OK;
}
