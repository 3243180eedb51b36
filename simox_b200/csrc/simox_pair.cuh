// simox_pair.cuh -- pieces shared by the pair passes (pair.cu: full lists,
// per-atom ownership; pair_half.cu: half lists with fixed-point scatter):
// the reference's pair forms in FP64 and FP32, the embedding, the minimum
// image, the skin-filter constants and the packed-FP32 pair function with its
// folded per-species constants.  Internal to libsimox_b200.so.
#pragma once

#include "simox_internal.cuh"
#include "simox_packed.cuh"

#include <algorithm>
#include <cmath>
#include <cstring>
#include <type_traits>

namespace sx {

// ---------------------------------------------------------------------------
// device math in R.  FP64: CUDA's exp / erfc / IEEE division.  FP32 (mixed
// path): the SFU exponential (ex2.approx on x*log2(e)), an approximate
// reciprocal, and erfc from the Chebyshev fit of Numerical Recipes (Press et
// al., "erfcc", fractional error < 1.2e-7 for all x >= 0), which shares the
// SFU exponential; tests/test_gpu_parity.py bounds the resulting force error.
template <typename R> __device__ __forceinline__ R dexp(R x);
template <> __device__ __forceinline__ double dexp<double>(double x) { return exp(x); }
template <> __device__ __forceinline__ float dexp<float>(float x) { return __expf(x); }
template <typename R> __device__ __forceinline__ R drcp(R x);
template <> __device__ __forceinline__ double drcp<double>(double x) { return 1.0 / x; }
template <> __device__ __forceinline__ float drcp<float>(float x) { return __fdividef(1.0f, x); }

// erfc(z) and exp(-z^2) for z >= 0
template <typename R> __device__ __forceinline__ void erfc_exp(R z, R& erfcv, R& ez2);
template <> __device__ __forceinline__ void erfc_exp<double>(double z, double& erfcv, double& ez2) {
    erfcv = erfc(z);
    ez2 = exp(-z * z);
}
template <> __device__ __forceinline__ void erfc_exp<float>(float z, float& erfcv, float& ez2) {
    const float t = __fdividef(1.0f, 1.0f + 0.5f * z);
    const float p = -1.26551223f + t * (1.00002368f + t * (0.37409196f + t * (0.09678418f +
                    t * (-0.18628806f + t * (0.27886807f + t * (-1.13520398f + t * (1.48851587f +
                    t * (-0.82215223f + t * 0.17087277f))))))));
    const float z2 = z * z;
    erfcv = t * __expf(p - z2);
    ez2 = __expf(-z2);
}

// Zhou term g = exp(-c(r/re - 1)) / (1 + (r/re - lam)^20) and dg/dr (eam.f90:16-23)
template <typename R>
__device__ __forceinline__ void zhou(R r, R ire, R c, R lam, R& g, R& dg) {
    const R rr = r * ire;
    const R t = rr - lam;
    const R t2 = t * t, t4 = t2 * t2, t8 = t4 * t4, t16 = t8 * t8;
    const R t19 = t16 * t2 * t, t20 = t19 * t;
    const R ex = dexp<R>(-c * (rr - R(1)));
    const R u = drcp<R>(R(1) + t20);
    g = ex * u;
    dg = g * ire * (-c - R(20) * t19 * u);
}
template <typename R>
__device__ __forceinline__ R zhou_val(R r, R ire, R c, R lam) {
    const R rr = r * ire;
    const R t = rr - lam;
    const R t2 = t * t, t4 = t2 * t2, t8 = t4 * t4, t16 = t8 * t8;
    const R t20 = t16 * t4;
    return dexp<R>(-c * (rr - R(1))) * drcp<R>(R(1) + t20);
}

// Embedding parameters (force.f90:256-351), by value into the kernel.
struct EmbedParams {
    double rho_e[3], rho_s[3], Fn[3][4], Fm[3][4], Fp[3][4], eta[3], Fe[3];
    double F[5][4], re[5], rmax[5];
};

__device__ __forceinline__ int embed(const EmbedParams& E, int s, double rho, double& F, double& dF) {
    double Fs = 0.0, d = 0.0, rr = 1.0;
    const double* cf = nullptr;
    if (s < 3) {
        double rho_n = 0.85 * E.rho_e[s], rho_0 = 1.15 * E.rho_e[s];
        if (rho < rho_n) { cf = E.Fn[s]; rr = rho_n; }
        else if (rho < E.rho_e[s]) { cf = E.Fm[s]; rr = E.rho_e[s]; }
        else if (rho < rho_0) { cf = E.Fp[s]; rr = E.rho_e[s]; }
        else if (rho > 1.0e-6) {
            double t = pow(rho / E.rho_s[s], E.eta[s]);
            double lt = log(t);
            Fs = E.Fe[s] * (1.0 - lt) * t;
            d = -E.Fe[s] * E.eta[s] * lt * t / rho;
        }
    } else if (s == 3) {
        int b = rho < E.rmax[0] ? 0 : rho < E.rmax[1] ? 1 : rho < E.rmax[2] ? 2 : rho < E.rmax[3] ? 3 : 4;
        cf = E.F[b]; rr = E.re[b];
    } else {
        F = 0.0; dF = 0.0;
        return 1;
    }
    if (cf) {
        double t = rho / rr - 1.0;
        Fs = cf[0] + cf[1] * t + cf[2] * (t * t) + cf[3] * (t * t * t);
        d = (cf[1] + cf[2] * 2.0 * t + cf[3] * 3.0 * (t * t)) / rr;
    }
    F = Fs; dF = d;
    return 0;
}

struct PairParams {
    double3 box, ibox;
    double a, kc, dr_rdf;
    int cap, n;
};

// separation with the reference's minimum image (force.f90:51-52)
__device__ __forceinline__ void min_image(double4 a, double4 b, const PairParams& P, double& dx, double& dy,
                                          double& dz) {
    dx = __dsub_rn(a.x, b.x);
    dy = __dsub_rn(a.y, b.y);
    dz = __dsub_rn(a.z, b.z);
    dx = __dsub_rn(dx, __dmul_rn(P.box.x, rint(dx * P.ibox.x)));
    dy = __dsub_rn(dy, __dmul_rn(P.box.y, rint(dy * P.ibox.y)));
    dz = __dsub_rn(dz, __dmul_rn(P.box.z, rint(dz * P.ibox.z)));
}

// list slot k of group g in a row (metals from the front, oxygen from the
// back); group 2 walks the whole row, nm = number of metal partners
__device__ __forceinline__ int row_slot(int g, int k, int cap, int nm = 0) {
    return g == 0 ? k : (g == 1 ? cap - 1 - k : (k < nm ? k : cap - 1 - (k - nm)));
}

constexpr int PK_THREADS = 256;

struct FilterParams {
    PairParams pp;
    double rcut2;
    float rcut2f, band;
    int3 nc;                 // reference cell grid (>= 3 per axis)
    int cap_s;
    float4 sh[kEntries];     // stencil position -> o * Lcs
};

// Density constants of one (X, Y) kind: FP32 filter in folded form
// (2^(k1 r + k0) / (1 + t^20), t = r ire + nlam, times fe), FP64 in the
// reference's form.
template <typename R>
struct DensC {
    R fe, ire, c, lam, k1, k0, nlam;
};

template <typename R>
__device__ __forceinline__ R dens_term(const DensC<R>& d, R r) {
    if constexpr (std::is_same<R, float>::value) {
        const float t = fmaf(r, d.ire, d.nlam);
        const float t2 = t * t, t4 = t2 * t2, t8 = t4 * t4, t16 = t8 * t8;
        const float ex = ex2_approx(fmaf(r, d.k1, d.k0));
        return d.fe * ex * rcp_approx(fmaf(t16, t4, 1.f));
    } else {
        return d.fe * zhou_val<double>(r, d.ire, d.c, d.lam);
    }
}

// Zhou term w(r) = Amp exp(-c (r/re - 1)) / (1 + (r/re - lam)^20) (eam.f90:16-31):
//   t = r ire + nlam, w = 2^(k1 r + k0) / (1 + t^20) with k0 = c log2(e) + log2|Amp|,
//   -dw/dr = w (m20 q + mc), q = t^19 / (1 + t^20), m20 = 20 s ire, mc = s c ire,
// s = sign(Amp).  Two terms share one reciprocal: 1/a = b / (ab), 1/b = a / (ab)
// (a, b <= 1 + 2e10 for r < Rcut = 10 A with the reference parameters).
struct ZhouC {
    float ire, nlam, k1, k0, m20, mc;
};

struct PackTab {
    ZhouC D, E, A, B;        // density at X from Y, density at Y from X, pair terms A and -B
    float cB;                // same-metal pairs: -B / fe (the B term has the density's shape)
    float ex1x, ex1y;        // -2 xi_X log2(e), -2 xi_Y log2(e)
    float txx, txy, x2x, x2y;  // 2 xi_X, 2 xi_Y, 2 xi_X^2, 2 xi_Y^2
    float Qx[5], Qy0, Qy3, Qy4;
    float kcZX, kcZY;        // kc Z_X, kc Z_Y
};


struct PackParams {
    float pa, na2l, tas, kc, inv_dr;   // p a, -a^2 log2(e), 2a/sqrt(pi), kc, 1/dr
    int cap;
    float4 sh[kEntries];
    PackTab tab[4];          // (metal, metal), (metal, O), (O, metal), (O, O)
};

__device__ __forceinline__ void zhou_parts(v2 r, const ZhouC& z, v2& t19, v2& den, v2& ex) {
    const v2 t = fma2(r, bc(z.ire), bc(z.nlam));
    const v2 t2 = t * t;
    const v2 t3 = t2 * t;
    const v2 t4 = t2 * t2;
    const v2 t8 = t4 * t4;
    const v2 t16 = t8 * t8;
    t19 = t16 * t3;
    den = fma2(t19, t, bc(1.f));
    ex = ex2(fma2(r, bc(z.k1), bc(z.k0)));
}
// -dw/dr given u = 1/den
__device__ __forceinline__ v2 zhou_nd(const ZhouC& z, v2 t19, v2 u, v2 ex) {
    const v2 w = ex * u;
    return w * fma2(t19 * u, bc(z.m20), bc(z.mc));
}

// f/r of one pair for the X-Y pair kind of T (force.f90:81-98, 101-140)
template <bool SAME, bool MHOMO>
__device__ __forceinline__ v2 pair_fs_pk(const PackTab& T, const PackParams& Q, v2 r2, v2 qb, v2 dFY, float dFX,
                                         float kcqa, float kcqaZY) {
    const v2 ir = rsqrt(r2);
    const v2 r = r2 * ir;
    const v2 ir2 = ir * ir;
    v2 eam;
    if (MHOMO) {
        v2 t19D, denD, exD, t19A, denA, exA;
        zhou_parts(r, T.D, t19D, denD, exD);
        zhou_parts(r, T.A, t19A, denA, exA);
        const v2 R = rcp(denD * denA);
        const v2 nD = zhou_nd(T.D, t19D, denA * R, exD);
        const v2 nA = zhou_nd(T.A, t19A, denD * R, exA);
        eam = fma2(dFY + bc(dFX + T.cB), nD, nA);
    } else {
        v2 t19A, denA, exA, t19B, denB, exB, t19D, denD, exD;
        zhou_parts(r, T.A, t19A, denA, exA);
        zhou_parts(r, T.B, t19B, denB, exB);
        const v2 R = rcp(denA * denB);
        eam = zhou_nd(T.A, t19A, denB * R, exA) + zhou_nd(T.B, t19B, denA * R, exB);
        zhou_parts(r, T.D, t19D, denD, exD);
        if (SAME) {
            eam = fma2(dFY + bc(dFX), zhou_nd(T.D, t19D, rcp(denD), exD), eam);
        } else {
            v2 t19E, denE, exE;
            zhou_parts(r, T.E, t19E, denE, exE);
            const v2 S = rcp(denD * denE);
            eam = fma2(bc(dFX), zhou_nd(T.D, t19D, denE * S, exD), eam);
            eam = fma2(dFY, zhou_nd(T.E, t19E, denD * S, exE), eam);
        }
    }
    // Ewald real space: kc qa qb (2a/sqrt(pi) r e^{-a^2 r^2} + erfc(a r)) / r^3
    const v2 kq = bc(kcqa) * qb;
    const v2 tt = rcp(fma2(r, bc(Q.pa), bc(1.f)));
    const v2 ez2 = ex2(r2 * bc(Q.na2l));
    const v2 ew = (kq * ez2) * (fma2(r, bc(Q.tas), tt * erfc_poly(tt)) * ir2);
    // CTIP Slater-1s terms
    const v2 eX = ex2(r * bc(T.ex1x));
    const v2 djfi = eX * fma2(fma2(r, bc(T.txx), bc(1.f)), ir2, bc(T.x2x));
    v2 ct;
    if (SAME) {
        const v2 QX = fma2(r, fma2(r, bc(T.Qx[2]), bc(T.Qx[1])), bc(T.Qx[0])) + ir * fma2(ir, bc(T.Qx[4]), bc(T.Qx[3]));
        const v2 dfifj = eX * QX;
        ct = fma2(qb, bc(T.kcZX), bc(kcqaZY)) * (dfifj - djfi) - kq * dfifj;
    } else {
        const v2 eY = ex2(r * bc(T.ex1y));
        const v2 difj = eY * fma2(fma2(r, bc(T.txy), bc(1.f)), ir2, bc(T.x2y));
        v2 dfifj = eX * fma2(ir, fma2(ir, bc(T.Qx[4]), bc(T.Qx[3])), bc(T.Qx[0]));
        dfifj = fma2(eY, fma2(ir, fma2(ir, bc(T.Qy4), bc(T.Qy3)), bc(T.Qy0)), dfifj);
        ct = fma2(bc(kcqaZY), dfifj - djfi, (qb * bc(T.kcZX)) * (dfifj - difj)) - kq * dfifj;
    }
    return ((eam + ew) + ct) * ir;
}

// host: folded constants of the packed pair function for species X, Y
static inline ZhouC zhou_const(double amp, double re, double c, double lam) {
    const double L2E = 1.4426950408889634;
    const double s = amp < 0.0 ? -1.0 : 1.0;
    ZhouC z;
    z.ire = (float)(1.0 / re);
    z.nlam = (float)(-lam);
    z.k1 = (float)(-c * L2E / re);
    z.k0 = amp != 0.0 ? (float)(c * L2E + std::log2(std::fabs(amp))) : -INFINITY;
    z.m20 = (float)(20.0 * s / re);
    z.mc = (float)(s * c / re);
    return z;
}

static inline PackTab pack_tab(const simox_potential& P, int X, int Y) {
    PackTab t;
    std::memset(&t, 0, sizeof(t));
    const bool mX = X < 3, mY = Y < 3;
    const simox_oxid& o = P.oxygn;
    auto dens = [&](int at, int from) {
        if (from < 3) {
            const simox_metl& e = P.eam[from];
            return zhou_const(e.f_e, e.r_e, e.beta, e.lambda);
        }
        const double re = at < 3 ? o.r_e[at] : o.r_e[3];     // eam.f90:196 / 297
        return zhou_const(o.fe, re, o.gamm, o.nu);
    };
    t.D = dens(X, Y);
    t.E = dens(Y, X);
    if (mX && mY) {                                          // METAL_HOMO eam.f90:29
        const simox_metl& e = P.eam[X];
        t.A = zhou_const(e.A, e.r_e, e.alpha, e.kappa);
        t.B = zhou_const(-e.B, e.r_e, e.beta, e.lambda);
        t.cB = (float)(-e.B / e.f_e);
    } else {                                                 // METAL_OXYGEN / OXYGEN_ONLY
        const int m = mX ? X : (mY ? Y : 3);
        t.A = zhou_const(o.A[m], o.r_e[m], o.alph[m], o.kapp[m]);
        t.B = zhou_const(-o.B[m], o.r_e[m], o.beta[m], o.lamb[m]);
    }
    const double L2E = 1.4426950408889634;
    const simox_potn& pX = P.param[X];
    const simox_potn& pY = P.param[Y];
    t.ex1x = (float)(-2.0 * pX.xi * L2E);
    t.ex1y = (float)(-2.0 * pY.xi * L2E);
    t.txx = (float)(2.0 * pX.xi);
    t.txy = (float)(2.0 * pY.xi);
    t.x2x = (float)(2.0 * pX.xi * pX.xi);
    t.x2y = (float)(2.0 * pY.xi * pY.xi);
    t.kcZX = (float)(SX_KC * pX.Z);
    t.kcZY = (float)(SX_KC * pY.Z);
    const double* f = pX.fafb[Y];
    if (X == Y) {       // force.f90:111-118
        const double xi = pX.xi;
        t.Qx[0] = (float)(2 * xi * f[1] - f[2]);
        t.Qx[1] = (float)(2 * xi * f[2] - 2 * f[3]);
        t.Qx[2] = (float)(2 * xi * f[3]);
        t.Qx[3] = (float)(2 * xi);
        t.Qx[4] = 1.f;
    } else {            // force.f90:130-133
        t.Qx[0] = (float)(2 * pX.xi * f[0]);
        t.Qx[3] = (float)(2 * pX.xi * f[2]);
        t.Qx[4] = (float)f[2];
        t.Qy0 = (float)(2 * pY.xi * f[1]);
        t.Qy3 = (float)(2 * pY.xi * f[3]);
        t.Qy4 = (float)f[3];
    }
    return t;
}

__device__ __forceinline__ void pair_energy_fp64(const PairTab<double>& T, double r, double ir, double qa, double qb,
                                                 double a, double& ep, double& ed, double& ec) {
    ep += T.p_A * zhou_val<double>(r, T.p_inv_re, T.p_alpha, T.p_kappa) -
          T.p_B * zhou_val<double>(r, T.p_inv_re, T.p_beta, T.p_lambda);   // eam.f90 phi
    ed += qa * qb * erfc(a * r) * ir;                                       // force.f90:94
    const double eX = exp(-2.0 * T.xi_x * r), eY = exp(-2.0 * T.xi_y * r);
    const double jfi = -eX * (T.xi_x + ir);
    const double ifj = -eY * (T.xi_y + ir);
    const double fifj = -eX * (T.Px[0] + r * (T.Px[1] + r * (T.Px[2] + r * T.Px[3])) + T.Px[4] * ir) -
                        eY * (T.Py[0] + T.Py[4] * ir);
    ec += qa * T.Z_y * (jfi - fifj) + qb * T.Z_x * (ifj - fifj) + qa * qb * fifj;   // force.f90:135-138
}

static inline EmbedParams embed_params(const simox_potential& P) {
    EmbedParams E;
    std::memset(&E, 0, sizeof(E));
    for (int s = 0; s < 3; s++) {
        const simox_metl& e = P.eam[s];
        E.rho_e[s] = e.rho_e; E.rho_s[s] = e.rho_s; E.eta[s] = e.eta; E.Fe[s] = e.Fe;
        for (int k = 0; k < 4; k++) { E.Fn[s][k] = e.Fn[k]; E.Fm[s][k] = e.Fm[k]; E.Fp[s][k] = e.Fp[k]; }
    }
    const simox_oxid& o = P.oxygn;
    const double* Fb[5] = {o.F0, o.F1, o.F2, o.F3, o.F4};
    for (int b = 0; b < 5; b++) {
        for (int k = 0; k < 4; k++) E.F[b][k] = Fb[b][k];
        E.re[b] = o.re[b]; E.rmax[b] = o.rmax[b];
    }
    return E;
}

static inline PairParams pair_params(const simox_ctx* c) {
    PairParams P;
    P.box = make_double3(c->box[0], c->box[1], c->box[2]);
    P.ibox = make_double3(c->inv_box[0], c->inv_box[1], c->inv_box[2]);
    P.a = c->a;
    P.kc = SX_KC;
    P.dr_rdf = c->dr_rdf;
    P.cap = c->nnb_cap;
    P.n = c->n;
    return P;
}

static inline int pair_grid(simox_ctx* c) {
    int wpb = PK_THREADS / 32;
    int need = (c->n + wpb - 1) / wpb;
    int lim = num_sms(c) * 8;
    return need < lim ? (need > 0 ? need : 1) : lim;
}

// Rounding bound of the FP32 r2 of a listed pair near the cutoff.  Offsets
// |off| <= A = Lcs/2 + skin/2 (+ slack) are rounded once (u = 2^-24), their
// difference once, o*Lcs once and the sum once: |err dx| <= u (6A + 2 Lcs);
// r2 = dx^2 + dy^2 + dz^2 with two fused steps adds <= 3u r2.  The band is
// four times that bound at r = Rcut.
static inline float filter_band(const simox_ctx* c) {
    const double u = std::ldexp(1.0, -24);
    double lmax = 0.0;
    for (int d = 0; d < 3; d++) lmax = std::max(lmax, c->lcs[d]);
    const double A = 0.5 * lmax + 0.5 * c->skin + 1.0e-3;
    const double e = u * (6.0 * A + 2.0 * lmax);
    const double bound = 2.0 * std::sqrt(3.0) * c->rcut * e + 3.0 * e * e + 3.0 * u * c->rcut2 * 1.01;
    return (float)(4.0 * bound);
}

// skin stencil position e = (dk+1)*9 + (dj+1)*3 + (di+1) -> o * Lcs
static inline void stencil_shifts(const simox_ctx* c, float4* sh) {
    for (int e = 0; e < kEntries; e++) {
        const int di = e % 3 - 1, dj = (e / 3) % 3 - 1, dk = e / 9 - 1;
        sh[e] = make_float4((float)(di * c->lcs[0]), (float)(dj * c->lcs[1]), (float)(dk * c->lcs[2]), 0.f);
    }
}

}  // namespace sx
