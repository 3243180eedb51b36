// pair.cu -- FORCE (force.f90:3-361) as two passes over the full neighbour list.
//
//  pass 1 (eam_density): rho_X = sum_Y f_{Y->X}(r) (force.f90:84-85), then the
//          embedding F(rho), F'(rho) of force.f90:256-351 per atom (FP64).
//  pass 2 (pair_forces): per pair the EAM pair and density forces
//          (force.f90:89-91, 349, 353-358 folded into -F'_X dD_X - F'_Y dD_Y),
//          the Ewald real-space term (force.f90:94-98) and the CTIP Slater
//          terms (force.f90:101-140); energies and the RDF histogram.
//
// One warp owns one atom (lanes stride over its neighbour row, then a warp
// reduction), so every force is written once and no float atomics are used.
// Precision: R = double (FP64 path) or float (mixed path: per-pair terms in
// FP32 from an FP64 separation; per-atom sums, energies in FP64).
#include "simox_internal.cuh"

#include <cmath>
#include <cstring>

namespace sx {

// ---------------------------------------------------------------------------
// host: uniform tables from the reference parameter set
template <typename R>
static void fill_tab(const simox_potential& P, PairTab<R>* T) {
    for (int X = 0; X < kSpecies; X++)
        for (int Y = 0; Y < kSpecies; Y++) {
            PairTab<R> t;
            std::memset(&t, 0, sizeof(t));
            const bool mX = X < 3, mY = Y < 3;
            t.valid = !(mX && mY && X != Y);
            const simox_oxid& o = P.oxygn;
            // density at X contributed by Y (eam.f90: metal ftn / oxygen exp_g form)
            auto dens = [&](int at, int from, R& fe, R& ire, R& cc, R& lam) {
                if (from < 3) {
                    const simox_metl& e = P.eam[from];
                    fe = (R)e.f_e; ire = (R)(1.0 / e.r_e); cc = (R)e.beta; lam = (R)e.lambda;
                } else {
                    double re = at < 3 ? o.r_e[at] : o.r_e[3];   // eam.f90:196 / 297
                    fe = (R)o.fe; ire = (R)(1.0 / re); cc = (R)o.gamm; lam = (R)o.nu;
                }
            };
            dens(X, Y, t.d_fe, t.d_inv_re, t.d_c, t.d_lam);
            dens(Y, X, t.e_fe, t.e_inv_re, t.e_c, t.e_lam);
            // pair phi
            if (mX && mY) {
                const simox_metl& e = P.eam[X];                  // METAL_HOMO eam.f90:29
                t.p_inv_re = (R)(1.0 / e.r_e); t.p_A = (R)e.A; t.p_alpha = (R)e.alpha; t.p_kappa = (R)e.kappa;
                t.p_B = (R)e.B; t.p_beta = (R)e.beta; t.p_lambda = (R)e.lambda;
            } else {
                int m = mX ? X : (mY ? Y : 3);                   // METAL_OXYGEN / OXYGEN_ONLY
                t.p_inv_re = (R)(1.0 / o.r_e[m]); t.p_A = (R)o.A[m]; t.p_alpha = (R)o.alph[m];
                t.p_kappa = (R)o.kapp[m]; t.p_B = (R)o.B[m]; t.p_beta = (R)o.beta[m]; t.p_lambda = (R)o.lamb[m];
            }
            // CTIP
            const simox_potn& pX = P.param[X];
            const simox_potn& pY = P.param[Y];
            t.xi_x = (R)pX.xi; t.xi_y = (R)pY.xi; t.Z_x = (R)pX.Z; t.Z_y = (R)pY.Z;
            const double* f = pX.fafb[Y];
            if (X == Y) {
                double xi = pX.xi;
                // fifj = -e (1 + f2 r + f3 r^2 + f4 r^3)              force.f90:107-110
                t.Px[0] = 1; t.Px[1] = (R)f[1]; t.Px[2] = (R)f[2]; t.Px[3] = (R)f[3]; t.Px[4] = 0;
                // dfifj = e((2xi r+1)(1/r^2+f2/r+f3+f4 r) - (f2/r+2f3+3f4 r)) force.f90:111-118
                t.Qx[0] = (R)(2 * xi * f[1] - f[2]); t.Qx[1] = (R)(2 * xi * f[2] - 2 * f[3]);
                t.Qx[2] = (R)(2 * xi * f[3]); t.Qx[3] = (R)(2 * xi); t.Qx[4] = 1;
                // CTIP_SOLVER: -e (1 + xr(f2 + xr(f3 + xr f4)))/r, xr = xi r  ctip.f90:91-93
                t.Sx[0] = 1; t.Sx[1] = (R)(f[1] * xi); t.Sx[2] = (R)(f[2] * xi * xi); t.Sx[3] = (R)(f[3] * xi * xi * xi);
            } else {
                double xx = pX.xi, xy = pY.xi;
                // fifj = -f1 eX - f2 eY - f3 eX/r - f4 eY/r            force.f90:126-129
                t.Px[0] = (R)f[0]; t.Px[4] = (R)f[2];
                t.Py[0] = (R)f[1]; t.Py[4] = (R)f[3];
                // dfifj = 2xX f1 eX + 2xY f2 eY + f3 eX(1+2xX r)/r^2 + f4 eY(1+2xY r)/r^2  force.f90:130-133
                t.Qx[0] = (R)(2 * xx * f[0]); t.Qx[3] = (R)(2 * xx * f[2]); t.Qx[4] = (R)f[2];
                t.Qy[0] = (R)(2 * xy * f[1]); t.Qy[3] = (R)(2 * xy * f[3]); t.Qy[4] = (R)f[3];
                // CTIP_SOLVER: -eX(f1 + f3/r) - eY(f2 + f4/r)          ctip.f90:97-100
                t.Sx[0] = (R)f[2]; t.Sx[1] = (R)f[0];
                t.Sy[0] = (R)f[3]; t.Sy[1] = (R)f[1];
            }
            T[X * kSpecies + Y] = t;
        }
}

int build_pair_tables(simox_ctx* c) {
    PairTab<double> td[kSpecies * kSpecies];
    PairTab<float> tf[kSpecies * kSpecies];
    fill_tab<double>(c->pot, td);
    fill_tab<float>(c->pot, tf);
    cudaError_t e1 = cudaMemcpyAsync(c->tab_d, td, sizeof(td), cudaMemcpyHostToDevice, c->stream);
    cudaError_t e2 = cudaMemcpyAsync(c->tab_f, tf, sizeof(tf), cudaMemcpyHostToDevice, c->stream);
    if (e1 != cudaSuccess || e2 != cudaSuccess) return SIMOX_E_CUDA;
    return cuda_status(cudaStreamSynchronize(c->stream));
}

// ---------------------------------------------------------------------------
// device math in R
template <typename R> __device__ __forceinline__ R dexp(R x);
template <> __device__ __forceinline__ double dexp<double>(double x) { return exp(x); }
template <> __device__ __forceinline__ float dexp<float>(float x) { return expf(x); }
template <typename R> __device__ __forceinline__ R derfc(R x);
template <> __device__ __forceinline__ double derfc<double>(double x) { return erfc(x); }
template <> __device__ __forceinline__ float derfc<float>(float x) { return erfcf(x); }
template <typename R> __device__ __forceinline__ R drcp(R x);
template <> __device__ __forceinline__ double drcp<double>(double x) { return 1.0 / x; }
template <> __device__ __forceinline__ float drcp<float>(float x) { return __fdividef(1.0f, x); }

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

constexpr int PK_THREADS = 256;

// pass 1 -------------------------------------------------------------------
template <typename R>
__global__ void __launch_bounds__(PK_THREADS)
    density_kernel(PairParams P, const PairTab<R>* __restrict__ tab, const double4* __restrict__ xq,
                   const int* __restrict__ ts, const int* __restrict__ nn, const unsigned* __restrict__ nbr,
                   EmbedParams E, double* __restrict__ rho_s, double* __restrict__ dF_s,
                   double* __restrict__ acc, int* __restrict__ status, int eflag) {
    __shared__ PairTab<R> st[kSpecies * kSpecies];
    __shared__ double red[PK_THREADS / 32];
    for (int k = threadIdx.x; k < kSpecies * kSpecies; k += blockDim.x) st[k] = tab[k];
    __syncthreads();
    const int lane = threadIdx.x & 31;
    const int wpb = blockDim.x >> 5;
    double egroup = 0.0;
    int bad = 0;
    for (int X = blockIdx.x * wpb + (threadIdx.x >> 5); X < P.n; X += gridDim.x * wpb) {
        const double4 xa = xq[X];
        const int sX = ts[X];
        const int m = nn[X];
        const unsigned* row = nbr + (size_t)X * P.cap;
        double rho = 0.0;
        for (int k = lane; k < m; k += 32) {
            const int Y = (int)(row[k] & kIdxMask);
            const double4 xb = xq[Y];
            const int sY = ts[Y];
            if (sX >= kSpecies || sY >= kSpecies) { bad |= ST_UNKNOWN_PAIR; continue; }
            double dx, dy, dz;
            min_image(xa, xb, P, dx, dy, dz);
            const R r2 = (R)__dadd_rn(__dadd_rn(__dmul_rn(dx, dx), __dmul_rn(dy, dy)), __dmul_rn(dz, dz));
            const R r = sqrt(r2);
            const PairTab<R>& T = st[sX * kSpecies + sY];
            if (!T.valid) bad |= ST_UNSUPPORTED;
            rho += (double)(T.d_fe * zhou_val<R>(r, T.d_inv_re, T.d_c, T.d_lam));
        }
        rho = warp_sum(rho);
        if (lane == 0) {
            double F, dF;
            if (embed(E, sX, rho, F, dF)) bad |= ST_UNKNOWN_ELEMENT;
            rho_s[X] = rho;
            dF_s[X] = dF;
            egroup += F;
        }
    }
    if (bad) atomicOr(status, bad);
    if (eflag) block_add<PK_THREADS>(egroup, acc, A_EGROUP, red);
}

// pass 2 -------------------------------------------------------------------
template <typename R, bool EFLAG, bool RDF>
__global__ void __launch_bounds__(PK_THREADS)
    force_kernel(PairParams P, const PairTab<R>* __restrict__ tab, const double4* __restrict__ xq,
                 const int* __restrict__ ts, const int* __restrict__ nn, const unsigned* __restrict__ nbr,
                 const double* __restrict__ dF_s, const int* __restrict__ sorted, double* __restrict__ f,
                 double* __restrict__ acc, int* __restrict__ rdf, int* __restrict__ status) {
    __shared__ PairTab<R> st[kSpecies * kSpecies];
    __shared__ double red[PK_THREADS / 32];
    constexpr int NB = SIMOX_NRDF + 2;
    __shared__ int hist[RDF ? kSpecies * kSpecies * NB : 1];
    for (int k = threadIdx.x; k < kSpecies * kSpecies; k += blockDim.x) st[k] = tab[k];
    if (RDF)
        for (int k = threadIdx.x; k < kSpecies * kSpecies * NB; k += blockDim.x) hist[k] = 0;
    __syncthreads();
    const int lane = threadIdx.x & 31;
    const int wpb = blockDim.x >> 5;
    const R a = (R)P.a;
    const R two_a_sqrtpi = (R)(2.0 * P.a / SX_SQRTPI);
    const R kc = (R)P.kc;
    double ep = 0.0, ed = 0.0, ec = 0.0;
    int bad = 0;
    for (int X = blockIdx.x * wpb + (threadIdx.x >> 5); X < P.n; X += gridDim.x * wpb) {
        const double4 xa = xq[X];
        const int sX = ts[X];
        const R qa = (R)xa.w;
        const R dFX = (R)dF_s[X];
        const int m = nn[X];
        const unsigned* row = nbr + (size_t)X * P.cap;
        double fx = 0.0, fy = 0.0, fz = 0.0;
        for (int k = lane; k < m; k += 32) {
            const unsigned ent = row[k];
            const int Y = (int)(ent & kIdxMask);
            const double4 xb = xq[Y];
            const int sY = ts[Y];
            if (sX >= kSpecies || sY >= kSpecies) { bad |= ST_UNKNOWN_PAIR; continue; }
            double dx, dy, dz;
            min_image(xa, xb, P, dx, dy, dz);
            const double r2d = __dadd_rn(__dadd_rn(__dmul_rn(dx, dx), __dmul_rn(dy, dy)), __dmul_rn(dz, dz));
            const R rx = (R)dx, ry = (R)dy, rz = (R)dz;
            const R r2 = (R)r2d;
            const R r = sqrt(r2);
            const R ir = drcp<R>(r);
            const R ir2 = ir * ir;
            const PairTab<R>& T = st[sX * kSpecies + sY];
            const R qb = (R)xb.w;
            const R dFY = (R)dF_s[Y];
            // EAM (eam.f90 pair forms; force.f90:81-91, 349, 356)
            R gD, dgD, gE, dgE, gA, dgA, gB, dgB;
            zhou<R>(r, T.d_inv_re, T.d_c, T.d_lam, gD, dgD);
            zhou<R>(r, T.e_inv_re, T.e_c, T.e_lam, gE, dgE);
            zhou<R>(r, T.p_inv_re, T.p_alpha, T.p_kappa, gA, dgA);
            zhou<R>(r, T.p_inv_re, T.p_beta, T.p_lambda, gB, dgB);
            const R dphi = T.p_A * dgA - T.p_B * dgB;
            R fs = -(dphi + dFX * T.d_fe * dgD + dFY * T.e_fe * dgE) * ir;
            // Ewald real space (force.f90:94-98)
            const R ar = a * r;
            const R erfcv = derfc<R>(ar);
            const R ea = dexp<R>(-ar * ar);
            fs += kc * qa * qb * (two_a_sqrtpi * r * ea + erfcv) * ir2 * ir;
            // CTIP (force.f90:101-140)
            const R eX = dexp<R>(R(-2) * T.xi_x * r);
            const R eY = dexp<R>(R(-2) * T.xi_y * r);
            const R djfi = eX * (R(2) * T.xi_x * T.xi_x + (R(1) + R(2) * T.xi_x * r) * ir2);
            const R difj = eY * (R(2) * T.xi_y * T.xi_y + (R(1) + R(2) * T.xi_y * r) * ir2);
            const R QX = T.Qx[0] + r * (T.Qx[1] + r * T.Qx[2]) + ir * (T.Qx[3] + ir * T.Qx[4]);
            const R QY = T.Qy[0] + r * (T.Qy[1] + r * T.Qy[2]) + ir * (T.Qy[3] + ir * T.Qy[4]);
            const R dfifj = eX * QX + eY * QY;
            const R ZX = T.Z_x, ZY = T.Z_y;
            fs += kc * ((qa * ZY + qb * ZX - qa * qb) * dfifj - qa * ZY * djfi - qb * ZX * difj) * ir;
            fx += (double)(rx * fs);
            fy += (double)(ry * fs);
            fz += (double)(rz * fs);
            if (!T.valid) bad |= ST_UNSUPPORTED;
            if (EFLAG) {
                ep += (double)(T.p_A * gA - T.p_B * gB);
                ed += (double)(qa * qb * erfcv * ir);
                const R jfi = -eX * (T.xi_x + ir);
                const R ifj = -eY * (T.xi_y + ir);
                const R PX = T.Px[0] + r * (T.Px[1] + r * (T.Px[2] + r * T.Px[3])) + T.Px[4] * ir;
                const R PY = T.Py[0] + r * (T.Py[1] + r * (T.Py[2] + r * T.Py[3])) + T.Py[4] * ir;
                const R fifj = -(eX * PX + eY * PY);
                ec += (double)(qa * ZY * (jfi - fifj) + qb * ZX * (ifj - fifj) + qa * qb * fifj);
            }
            if (RDF && (ent & kIsA)) {
                int bin;
                if (sizeof(R) == 8) bin = __double2int_rz(__ddiv_rn(__dsqrt_rn(r2d), P.dr_rdf));  // INT(r/dr)
                else bin = (int)((float)r * (float)(1.0 / P.dr_rdf));
                bin = min(max(bin, 0), NB - 1);
                atomicAdd(&hist[(sX + kSpecies * sY) * NB + bin], 2);
            }
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
    if (bad) atomicOr(status, bad);
    if (EFLAG) {
        block_add<PK_THREADS>(0.5 * ep, acc, A_EPAIR, red);
        block_add<PK_THREADS>(0.5 * ed, acc, A_EDIR, red);
        block_add<PK_THREADS>(0.5 * ec, acc, A_ECTIP, red);
    }
    if (RDF) {
        __syncthreads();
        for (int k = threadIdx.x; k < kSpecies * kSpecies * NB; k += blockDim.x) {
            int v = hist[k];
            if (v) {
                int pr = k / NB, bin = k % NB;
                int si = pr % kSpecies, sj = pr / kSpecies;
                atomicAdd(&rdf[si + 5 * sj + 25 * bin], v);
            }
        }
    }
}

static EmbedParams embed_params(const simox_potential& P) {
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

static PairParams pair_params(const simox_ctx* c) {
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

static int pair_grid(simox_ctx* c) {
    int wpb = PK_THREADS / 32;
    int need = (c->n + wpb - 1) / wpb;
    int lim = num_sms(c) * 8;
    return need < lim ? (need > 0 ? need : 1) : lim;
}

int eam_density(simox_ctx* c, bool eflag) {
    int st = ensure_list(c);
    if (st) return st;
    if (c->n == 0) return SIMOX_OK;
    PairParams P = pair_params(c);
    EmbedParams E = embed_params(c->pot);
    Launch L(c, "eam_density");
    if (c->precision == SIMOX_MIXED)
        density_kernel<float><<<pair_grid(c), PK_THREADS, 0, c->stream>>>(P, c->tab_f, c->xq_s, c->t_s, c->nn, c->nbr, E,
                                                                         c->rho_s, c->dF_s, c->acc, c->status, eflag);
    else
        density_kernel<double><<<pair_grid(c), PK_THREADS, 0, c->stream>>>(P, c->tab_d, c->xq_s, c->t_s, c->nn, c->nbr,
                                                                          E, c->rho_s, c->dF_s, c->acc, c->status,
                                                                          eflag);
    c->eam_valid = true;
    return check_launch(c);
}

template <typename R>
static void launch_force(simox_ctx* c, const PairTab<R>* tab, bool eflag, bool rdf) {
    PairParams P = pair_params(c);
    int g = pair_grid(c);
    if (eflag && rdf)
        force_kernel<R, true, true><<<g, PK_THREADS, 0, c->stream>>>(P, tab, c->xq_s, c->t_s, c->nn, c->nbr, c->dF_s,
                                                                     c->sorted, c->f, c->acc, c->rdf, c->status);
    else if (eflag)
        force_kernel<R, true, false><<<g, PK_THREADS, 0, c->stream>>>(P, tab, c->xq_s, c->t_s, c->nn, c->nbr, c->dF_s,
                                                                      c->sorted, c->f, c->acc, c->rdf, c->status);
    else if (rdf)
        force_kernel<R, false, true><<<g, PK_THREADS, 0, c->stream>>>(P, tab, c->xq_s, c->t_s, c->nn, c->nbr, c->dF_s,
                                                                      c->sorted, c->f, c->acc, c->rdf, c->status);
    else
        force_kernel<R, false, false><<<g, PK_THREADS, 0, c->stream>>>(P, tab, c->xq_s, c->t_s, c->nn, c->nbr, c->dF_s,
                                                                       c->sorted, c->f, c->acc, c->rdf, c->status);
}

int pair_forces(simox_ctx* c, bool eflag, bool rdf) {
    if (!c->eam_valid) return SIMOX_E_STATE;
    if (c->n == 0) return SIMOX_OK;
    Launch L(c, "pair_force");
    if (c->precision == SIMOX_MIXED) launch_force<float>(c, c->tab_f, eflag, rdf);
    else launch_force<double>(c, c->tab_d, eflag, rdf);
    return check_launch(c);
}

}  // namespace sx
