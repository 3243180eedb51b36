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
// Rows are grouped by partner species, and each group runs code specialised
// for its species pair: Al-Al needs two Zhou terms and one CTIP exponential,
// O-O three and one, Al-O four and two (the uniform form needs four and two).
// Precision: R = double (FP64 path) or float (mixed path: per-pair terms in
// FP32 from an FP64 separation; per-atom sums, energies in FP64).
#include "simox_pair.cuh"

#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstring>
#include <type_traits>

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
            double cPx[5], cPy[5], cQx[5], cQy[5], cSx[4], cSy[4];
            ctip_coefs<double>(pX.xi, pY.xi, X == Y, pX.fafb[Y], cPx, cPy, cQx, cQy, cSx, cSy);
            for (int k = 0; k < 5; k++) {
                t.Px[k] = (R)cPx[k]; t.Py[k] = (R)cPy[k]; t.Qx[k] = (R)cQx[k]; t.Qy[k] = (R)cQy[k];
            }
            for (int k = 0; k < 4; k++) { t.Sx[k] = (R)cSx[k]; t.Sy[k] = (R)cSy[k]; }
            T[X * kSpecies + Y] = t;
        }
}

int build_pair_tables(simox_ctx* c) {
    PairTab<double> td[kSpecies * kSpecies];
    PairTab<float> tf[kSpecies * kSpecies];
    fill_tab<double>(c->pot, td);
    fill_tab<float>(c->pot, tf);
    std::memcpy(c->h_tab_f, tf, sizeof(tf));
    cudaError_t e1 = cudaMemcpyAsync(c->tab_d, td, sizeof(td), cudaMemcpyHostToDevice, c->stream);
    cudaError_t e2 = cudaMemcpyAsync(c->tab_f, tf, sizeof(tf), cudaMemcpyHostToDevice, c->stream);
    if (e1 != cudaSuccess || e2 != cudaSuccess) return SIMOX_E_CUDA;
    return cuda_status(cudaStreamSynchronize(c->stream));
}



// pass 1 -------------------------------------------------------------------
template <typename R>
__global__ void __launch_bounds__(PK_THREADS)
    density_kernel(PairParams P, const PairTab<R>* __restrict__ tab, const double4* __restrict__ xq,
                   const int* __restrict__ ts, const int2* __restrict__ nn, const unsigned* __restrict__ nbr,
                   EmbedParams E, double* __restrict__ rho_s, double* __restrict__ dF_s, float* __restrict__ dF_f,
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
        const int2 m = nn[X];
        const unsigned* row = nbr + (size_t)X * P.cap;
        double rho = 0.0;
        if (sX < kSpecies) {
#pragma unroll 1
            for (int g = 0; g < 2; g++) {
                const int mg = g == 0 ? m.x : m.y;
                // partner species of the group: oxygen (3) for g = 1; metals for g = 0
                unsigned ent_n = lane < mg ? row[row_slot(g, lane, P.cap)] : 0u;
                double4 xb_n = lane < mg ? xq[ent_n & kIdxMask] : make_double4(0, 0, 0, 0);
                for (int k = lane; k < mg; k += 32) {
                    const int Y = (int)(ent_n & kIdxMask);
                    const double4 xb = xb_n;
                    if (k + 32 < mg) {
                        ent_n = row[row_slot(g, k + 32, P.cap)];
                        xb_n = xq[ent_n & kIdxMask];
                    }
                    const int sY = g == 1 ? 3 : ts[Y];
                    if (sY >= kSpecies) { bad |= ST_UNKNOWN_PAIR; continue; }
                    double dx, dy, dz;
                    min_image(xa, xb, P, dx, dy, dz);
                    const R r2 = (R)__dadd_rn(__dadd_rn(__dmul_rn(dx, dx), __dmul_rn(dy, dy)), __dmul_rn(dz, dz));
                    const R r = sqrt(r2);
                    const PairTab<R>& T = st[sX * kSpecies + sY];
                    if (!T.valid) bad |= ST_UNSUPPORTED;
                    rho += (double)(T.d_fe * zhou_val<R>(r, T.d_inv_re, T.d_c, T.d_lam));
                }
            }
        } else if (m.x + m.y > 0) {
            bad |= ST_UNKNOWN_PAIR;
        }
        rho = warp_sum(rho);
        if (lane == 0) {
            double F, dF;
            if (embed(E, sX, rho, F, dF)) bad |= ST_UNKNOWN_ELEMENT;
            rho_s[X] = rho;
            dF_s[X] = dF;
            dF_f[X] = (float)dF;
            egroup += F;
        }
    }
    if (bad) atomicOr(status, bad);
    if (eflag) block_add<PK_THREADS>(egroup, acc, A_EGROUP, red);
}

// Skin-mode list filter fused with pass 1.  Per atom X, the skin row (cutoff
// Rcut + skin) is tested against the reference's FP64 r2 < Rcut2
// (force.f90:51-54); kept partners are written, compacted with a warp ballot,
// to the exact row (same species grouping, stencil position kept) with bit
// 31 = "X is the reference's i" (Y's reference cell is one of the 13
// CELL_HIERARCHY cells of X's, or the same cell and X comes first), and their density terms are
// summed into rho_X; the embedding follows as in density_kernel.
//
// FP32 contexts decide membership from the 16-byte filter records: r2 from
// off_Y - off_X + o*Lcs in FP32, and only pairs whose FP32 r2 lies within the
// rounding bound `band` of Rcut^2 are re-tested with the FP64 positions.  FP64
// contexts test every pair in FP64.

// One group of X's skin row (G = 0: metal partners, row front; G = 1: oxygen
// partners, row back).  UNI: the partner species of the group is fixed (sYf),
// so its density constants sit in registers; otherwise they are looked up per
// entry.  Kept entries are compacted into X's exact row (same end of the row)
// with bit 31 = "X is the reference's i".  Returns the kept count.
template <typename R, int G, bool UNI>
__device__ __forceinline__ int filter_group(const FilterParams& F, const float4* ssh, const DensC<R>* dsh,
                                            const int* dflag, int sX, int sYf, const unsigned* __restrict__ sp,
                                            int mg, unsigned* __restrict__ dp, const float4& ra, unsigned wa, int xm,
                                            int ym, int zm, int oX, const double4& xa, int X,
                                            const double4* __restrict__ xq, const float4* __restrict__ rec,
                                            const int* __restrict__ order, double& rho, int& bad) {
    constexpr bool F32 = std::is_same<R, float>::value;
    const PairParams& P = F.pp;
    const int lane = threadIdx.x & 31;
    const unsigned lt = (1u << lane) - 1u;
    const int ax = wa & 511, ay = (wa >> 9) & 511, az = (wa >> 18) & 511;
    DensC<R> du{};
    if (UNI) {
        du = dsh[(sX << 3) | sYf];
        if (mg > 0) bad |= dflag[(sX << 3) | sYf];
    }
    auto ent = [&](int k) { return k < mg ? sp[G == 0 ? k : -k] : 0u; };
    unsigned E1 = ent(lane), E2 = ent(lane + 32);
    float4 rb1 = rec[E1 & kSkinIdxMask];
    double4 xb1 = F32 ? make_double4(0, 0, 0, 0) : xq[E1 & kSkinIdxMask];
    int out = 0;
    for (int base = 0; base < mg; base += 32) {
        const int k = base + lane;
        const unsigned e = E1;
        const float4 rb = rb1;
        const double4 xb = xb1;
        E1 = E2;
        rb1 = rec[E1 & kSkinIdxMask];
        if (!F32) xb1 = xq[E1 & kSkinIdxMask];
        E2 = ent(k + 64);
        const unsigned Y = e & kSkinIdxMask;
        const bool live = k < mg;
        bool acc;
        R r2;
        if constexpr (F32) {
            const float4 o = ssh[e >> kSkinCodeShift];
            const float dx = (rb.x - ra.x) + o.x, dy = (rb.y - ra.y) + o.y, dz = (rb.z - ra.z) + o.z;
            const float r2f = fmaf(dx, dx, fmaf(dy, dy, dz * dz));
            acc = live & (r2f < F.rcut2f);
            const bool inband = live & (fabsf(r2f - F.rcut2f) <= F.band);
            if (__any_sync(0xffffffffu, inband)) {
                if (inband) {
                    // within FP32 rounding of the cutoff: the reference's FP64 test
                    double ddx, ddy, ddz;
                    min_image(xq[X], xq[Y], P, ddx, ddy, ddz);
                    acc = __dadd_rn(__dadd_rn(__dmul_rn(ddx, ddx), __dmul_rn(ddy, ddy)), __dmul_rn(ddz, ddz)) <
                          F.rcut2;
                }
            }
            r2 = r2f;
        } else {
            double dx, dy, dz;
            min_image(xa, xb, P, dx, dy, dz);
            const double r2d = __dadd_rn(__dadd_rn(__dmul_rn(dx, dx), __dmul_rn(dy, dy)), __dmul_rn(dz, dz));
            acc = live & (r2d < F.rcut2);
            r2 = r2d;
        }
        // X is the reference's i: Y's reference cell is one of the 13 forward
        // cells of X's (cellsort.f90:18-30), or the same cell and X comes first
        const unsigned wb = __float_as_uint(rb.w);
        const int bx = wb & 511, by = (wb >> 9) & 511, bz = (wb >> 18) & 511;
        const bool same = ((wb ^ wa) & 0x07ffffffu) == 0u;
        int oY = 0x7fffffff;
        if (acc & same) oY = order[Y];
        const bool isa = (bz == zm) | ((bz == az) & ((by == ym) | ((by == ay) & ((bx == xm) | (same & (oX < oY))))));
        const unsigned mask = __ballot_sync(0xffffffffu, acc);
        const int pos = out + __popc(mask & lt);
        if (acc & (pos < P.cap)) dp[G == 0 ? pos : -pos] = e | ((unsigned)isa << 31);
        out += __popc(mask);
        // density of Y at X (force.f90:84-85)
        R r;
        if constexpr (F32) r = r2 * rsqrt_approx(r2);
        else r = sqrt(r2);
        R v;
        if (UNI) {
            v = dens_term<R>(du, r);
        } else {
            const int ti = (sX << 3) | (int)(wb >> 27);
            v = dens_term<R>(dsh[ti], r);
            bad |= acc ? dflag[ti] : 0;
        }
        rho += acc ? (double)v : 0.0;
    }
    return out;
}

// One atom of pass 1: filter X's skin row into its exact row, sum its density,
// embedding derivative and list statistics.
template <typename R>
__device__ __forceinline__ void filter_atom(const FilterParams& F, const float4* ssh, const DensC<R>* dsh,
                                            const int* dflag, int X, const double4* __restrict__ xq,
                                            const float4* __restrict__ rec, const int* __restrict__ order,
                                            const int2* __restrict__ nn_s, const unsigned* __restrict__ nbr_s,
                                            int2* __restrict__ nn, unsigned* __restrict__ nbr, const EmbedParams& E,
                                            double* __restrict__ rho_s, double* __restrict__ dF_s,
                                            float* __restrict__ dF_f, int* __restrict__ status, int& lmax,
                                            unsigned long long& ltot, int& bad, int g0) {
    constexpr bool F32 = std::is_same<R, float>::value;
    const PairParams& P = F.pp;
    const int lane = threadIdx.x & 31;
    const float4 ra = rec[X];
    const unsigned wa = __float_as_uint(ra.w);
    const int sX = (int)(wa >> 27);
    const int ax = wa & 511, ay = (wa >> 9) & 511, az = (wa >> 18) & 511;
    // the "-1" neighbours of X's reference cell on each axis (periodic)
    const int xm = ax == 0 ? F.nc.x - 1 : ax - 1;
    const int ym = ay == 0 ? F.nc.y - 1 : ay - 1;
    const int zm = az == 0 ? F.nc.z - 1 : az - 1;
    const int oX = order[X];
    const double4 xa = F32 ? make_double4(0, 0, 0, 0) : xq[X];
    const int2 ms = nn_s[X];
    const unsigned* srow = nbr_s + (size_t)X * F.cap_s;
    unsigned* row = nbr + (size_t)X * P.cap;
    double rho = 0.0;
    int out0, out1;
    if (g0 >= 0)
        out0 = filter_group<R, 0, true>(F, ssh, dsh, dflag, sX, g0, srow, ms.x, row, ra, wa, xm, ym, zm, oX, xa,
                                        X, xq, rec, order, rho, bad);
    else
        out0 = filter_group<R, 0, false>(F, ssh, dsh, dflag, sX, 0, srow, ms.x, row, ra, wa, xm, ym, zm, oX, xa,
                                         X, xq, rec, order, rho, bad);
    out1 = filter_group<R, 1, true>(F, ssh, dsh, dflag, sX, 3, srow + (F.cap_s - 1), ms.y, row + (P.cap - 1), ra,
                                    wa, xm, ym, zm, oX, xa, X, xq, rec, order, rho, bad);
    rho = warp_sum(rho);
    if (lane == 0) {
        const int tot = out0 + out1;
        if (tot > P.cap) {
            atomicOr(status, ST_NBR_OVERFLOW);
            nn[X] = make_int2(0, 0);
        } else {
            nn[X] = make_int2(out0, out1);
        }
        lmax = max(lmax, tot);
        ltot += (unsigned long long)tot;
        double Fe, dF;
        if (embed(E, sX, rho, Fe, dF)) bad |= ST_UNKNOWN_ELEMENT;
        rho_s[X] = rho;
        dF_s[X] = dF;
        dF_f[X] = (float)dF;
    }
}

template <typename R>
__global__ void __launch_bounds__(256)
    filter_density_kernel(FilterParams F, const PairTab<R>* __restrict__ tab, const double4* __restrict__ xq,
                          const float4* __restrict__ rec, const int* __restrict__ order,
                          const int2* __restrict__ nn_s, const unsigned* __restrict__ nbr_s, int2* __restrict__ nn,
                          unsigned* __restrict__ nbr, EmbedParams E, double* __restrict__ rho_s,
                          double* __restrict__ dF_s, float* __restrict__ dF_f, int* __restrict__ status,
                          int* __restrict__ nn_max, unsigned long long* __restrict__ nn_tot, int g0) {
    // density constants by (species X, species Y) with species in 3 bits (7:
    // unknown), and the status bits a pair of that kind raises
    __shared__ DensC<R> dsh[64];
    __shared__ int dflag[64];
    __shared__ float4 ssh[kEntries];
    for (int k = threadIdx.x; k < 64; k += blockDim.x) {
        const int a = k >> 3, b = k & 7;
        DensC<R> d{};
        int fl;
        if (a < kSpecies && b < kSpecies) {
            const PairTab<R>& T = tab[a * kSpecies + b];
            d.fe = T.d_fe; d.ire = T.d_inv_re; d.c = T.d_c; d.lam = T.d_lam;
            d.nlam = -T.d_lam;
            d.k1 = (R)(-1.4426950408889634) * T.d_c * T.d_inv_re;
            d.k0 = (R)1.4426950408889634 * T.d_c;
            fl = T.valid ? 0 : ST_UNSUPPORTED;
        } else {
            d.fe = 0; d.ire = 1; d.c = 0; d.lam = 0; d.nlam = 0; d.k1 = 0; d.k0 = 0;
            fl = ST_UNKNOWN_PAIR;
        }
        dsh[k] = d;
        dflag[k] = fl;
    }
    for (int k = threadIdx.x; k < kEntries; k += blockDim.x) ssh[k] = F.sh[k];
    __syncthreads();
    constexpr bool F32 = std::is_same<R, float>::value;
    const PairParams& P = F.pp;
    const int lane = threadIdx.x & 31, wpb = blockDim.x >> 5;
    int lmax = 0, bad = 0;
    unsigned long long ltot = 0;
    for (int X = blockIdx.x * wpb + (threadIdx.x >> 5); X < P.n; X += gridDim.x * wpb)
        filter_atom<R>(F, ssh, dsh, dflag, X, xq, rec, order, nn_s, nbr_s, nn, nbr, E, rho_s, dF_s, dF_f,
                              status, lmax, ltot, bad, g0);
    if (bad) atomicOr(status, bad);
    if (lane == 0) {
        if (lmax) atomicMax(nn_max, lmax);
        if (ltot) atomicAdd(nn_tot, ltot);
    }
}

// Egroup = sum_X F(rho_X) from stored densities (energy steps after a fused pass)
__global__ void __launch_bounds__(256)
    embed_energy_kernel(int n, const int* __restrict__ ts, const double* __restrict__ rho_s, EmbedParams E,
                        double* __restrict__ acc) {
    __shared__ double red[256 / 32];
    double eg = 0.0;
    const int X = blockIdx.x * blockDim.x + threadIdx.x;
    if (X < n) {
        double Fe, dF;
        embed(E, ts[X], rho_s[X], Fe, dF);
        eg = Fe;
    }
    block_add<256>(eg, acc, A_EGROUP, red);
}

// One pair's scalar force f/r on X (force.f90:81-98, 135-138), specialised on
//   SAME : the partner has X's species (one density function, one CTIP exponential)
//   MHOMO: same-species metals, whose pair B-term is the density shape (METAL_HOMO)
template <typename R, bool SAME, bool MHOMO, bool EFLAG>
__device__ __forceinline__ R pair_fs(const PairTab<R>& T, R r, R ir, R qa, R qb, R dFX, R dFY, R a,
                                     R two_a_sqrtpi, R kc, R& erfcv, double& ep, double& ed, double& ec) {
    const R ir2 = ir * ir;
    R fs;
    if (MHOMO) {
        R g, dg, gA, dgA;
        zhou<R>(r, T.d_inv_re, T.d_c, T.d_lam, g, dg);          // ftn, eam.f90:21-23
        zhou<R>(r, T.p_inv_re, T.p_alpha, T.p_kappa, gA, dgA);  // eam.f90:29-31
        fs = -(T.p_A * dgA - T.p_B * dg + (dFX + dFY) * T.d_fe * dg) * ir;
        if (EFLAG) ep += (double)(T.p_A * gA - T.p_B * g);
    } else {
        R gD, dgD, gA, dgA, gB, dgB, dgE;
        zhou<R>(r, T.d_inv_re, T.d_c, T.d_lam, gD, dgD);
        if (SAME) {
            dgE = dgD;
        } else {
            R gE;
            zhou<R>(r, T.e_inv_re, T.e_c, T.e_lam, gE, dgE);
        }
        zhou<R>(r, T.p_inv_re, T.p_alpha, T.p_kappa, gA, dgA);
        zhou<R>(r, T.p_inv_re, T.p_beta, T.p_lambda, gB, dgB);
        fs = -(T.p_A * dgA - T.p_B * dgB + dFX * T.d_fe * dgD + dFY * T.e_fe * dgE) * ir;
        if (EFLAG) ep += (double)(T.p_A * gA - T.p_B * gB);
    }
    // Ewald real space (force.f90:94-98)
    R ea;
    erfc_exp<R>(a * r, erfcv, ea);
    fs += kc * qa * qb * (two_a_sqrtpi * r * ea + erfcv) * ir2 * ir;
    // CTIP (force.f90:101-140)
    const R eX = dexp<R>(R(-2) * T.xi_x * r);
    const R eY = SAME ? eX : dexp<R>(R(-2) * T.xi_y * r);
    const R djfi = eX * (R(2) * T.xi_x * T.xi_x + (R(1) + R(2) * T.xi_x * r) * ir2);
    const R difj = SAME ? djfi : eY * (R(2) * T.xi_y * T.xi_y + (R(1) + R(2) * T.xi_y * r) * ir2);
    const R QX = T.Qx[0] + r * (T.Qx[1] + r * T.Qx[2]) + ir * (T.Qx[3] + ir * T.Qx[4]);
    R dfifj = eX * QX;
    if (!SAME) dfifj += eY * (T.Qy[0] + ir * (T.Qy[3] + ir * T.Qy[4]));
    const R ZX = T.Z_x, ZY = T.Z_y;
    fs += kc * ((qa * ZY + qb * ZX - qa * qb) * dfifj - qa * ZY * djfi - qb * ZX * difj) * ir;
    if (EFLAG) {
        ed += (double)(qa * qb * erfcv * ir);
        const R jfi = -eX * (T.xi_x + ir);
        const R ifj = SAME ? jfi : -eY * (T.xi_y + ir);
        R fifj = -eX * (T.Px[0] + r * (T.Px[1] + r * (T.Px[2] + r * T.Px[3])) + T.Px[4] * ir);
        if (!SAME) fifj -= eY * (T.Py[0] + T.Py[4] * ir);
        ec += (double)(qa * ZY * (jfi - fifj) + qb * ZX * (ifj - fifj) + qa * qb * fifj);
    }
    return fs;
}

// One group of X's row with a fixed specialisation.
// F' of a partner: the FP32 copy on the mixed path, FP64 otherwise
template <typename R> __device__ __forceinline__ R dFY_of(const double* dF, const float* dFf, int Y);
template <> __device__ __forceinline__ double dFY_of<double>(const double* dF, const float*, int Y) { return dF[Y]; }
template <> __device__ __forceinline__ float dFY_of<float>(const double*, const float* dFf, int Y) { return dFf[Y]; }

template <typename R, bool SAME, bool MHOMO, bool EFLAG, bool RDF>
__device__ __forceinline__ void force_group(const PairParams& P, const PairTab<R>* st, const unsigned* row, int g,
                                            int mg, int lane, const double4& xa, int sX, int sY_fixed, R qa, R dFX,
                                            const double4* __restrict__ xq, const int* __restrict__ ts,
                                            const double* __restrict__ dF_s, const float* __restrict__ dF_f,
                                            double& fx, double& fy, double& fz,
                                            double& ep, double& ed, double& ec, int* hist, int& bad) {
    constexpr int NB = SIMOX_NRDF + 2;
    const R a = (R)P.a;
    const R two_a_sqrtpi = (R)(2.0 * P.a / SX_SQRTPI);
    const R kc = (R)P.kc;
    const int nm = g == 2 ? sY_fixed : 0;
    if (g == 2) sY_fixed = -1;
    // software pipeline: the next iteration's list entry, position and F' are
    // loaded before this iteration's arithmetic
    unsigned ent_n = 0;
    double4 xb_n = make_double4(0, 0, 0, 0);
    R dFY_n = 0;
    if (lane < mg) {
        ent_n = row[row_slot(g, lane, P.cap, nm)];
        xb_n = xq[ent_n & kIdxMask];
        dFY_n = dFY_of<R>(dF_s, dF_f, (int)(ent_n & kIdxMask));
    }
    for (int k = lane; k < mg; k += 32) {
        const unsigned ent = ent_n;
        const int Y = (int)(ent & kIdxMask);
        const double4 xb = xb_n;
        const R dFY = dFY_n;
        if (k + 32 < mg) {
            ent_n = row[row_slot(g, k + 32, P.cap, nm)];
            xb_n = xq[ent_n & kIdxMask];
            dFY_n = dFY_of<R>(dF_s, dF_f, (int)(ent_n & kIdxMask));
        }
        const int sY = sY_fixed >= 0 ? sY_fixed : ts[Y];
        if (sY >= kSpecies) { bad |= ST_UNKNOWN_PAIR; continue; }
        if (MHOMO && sY != sX) { bad |= ST_UNSUPPORTED; continue; }
        double dx, dy, dz;
        min_image(xa, xb, P, dx, dy, dz);
        const double r2d = __dadd_rn(__dadd_rn(__dmul_rn(dx, dx), __dmul_rn(dy, dy)), __dmul_rn(dz, dz));
        R r, ir;
        if (sizeof(R) == 8) { r = (R)sqrt(r2d); ir = R(1) / r; }
        else { ir = (R)rsqrtf((float)r2d); r = (R)r2d * ir; }
        const PairTab<R>& T = st[sX * kSpecies + sY];
        R erfcv;
        const R fs = pair_fs<R, SAME, MHOMO, EFLAG>(T, r, ir, qa, (R)xb.w, dFX, dFY, a, two_a_sqrtpi, kc, erfcv, ep,
                                                    ed, ec);
        // f_X += rx * fs, accumulated in FP64 on the FP64 separation
        const double fsd = (double)fs;
        fx = fma(fsd, dx, fx);
        fy = fma(fsd, dy, fy);
        fz = fma(fsd, dz, fz);
        if (RDF && (ent & kIsA)) {
            int bin;
            if (sizeof(R) == 8) bin = __double2int_rz(__ddiv_rn(__dsqrt_rn(r2d), P.dr_rdf));  // INT(r/dr)
            else bin = (int)((float)r * (float)(1.0 / P.dr_rdf));
            bin = min(max(bin, 0), NB - 1);
            atomicAdd(&hist[(sX + kSpecies * sY) * NB + bin], 2);
        }
    }
}

// Skin-mode FP32 force pass (one metal species plus oxygen, no energies).
//
// The separation comes from the force records, x_X - x_Y = off_X - off_Y -
// o * Lcs (o: the entry's stencil position), so no FP64 minimum image is
// needed.  Each thread evaluates two entries of X's row at once (entries k and
// k + 32 of a 64-entry batch) as the halves of packed FP32 values, so every
// FP32 step of the pair function is one FFMA2/FMUL2/FADD2 for both
// (simox_packed.cuh).  The pair function is force.f90:81-98 and 101-140 with
// the constants folded per species pair (PackTab); each lane sums its share
// of f_X in compensated FP32 (hi + lo, TwoSum) and the lanes' sums are added
// in FP64.
//


// Cell-tiled force pass.  Atoms are in skin-cell order, and every entry of a
// row names its partner's cell by the stencil position e (0..26) relative to
// the atom's own cell.  One CTA takes the atoms of one skin cell (or a part
// of it) and first copies the records and F' of the 27 cells around it into
// shared memory (cp.async); a row entry then resolves with one table lookup
// (the stencil shift o_e * Lcs and the index delta of cell e's tile) and two
// shared loads.  A neighbourhood larger than the tile reads the same data
// from global memory instead.
constexpr int kTileThreads = 256;
constexpr int kTileBlocks = 2;             // resident CTAs per SM (tile ~110 KB each)
constexpr int kTileCap = 5500;             // records per tile (16 B record + 4 B F')
constexpr int kSelfEntry = 13;             // stencil position (0, 0, 0)

template <bool SAME, bool MHOMO, bool RDF, bool TILED, int TI>
__device__ __forceinline__ void force_batch_tile(const PackParams& Q, const float4* etab, const float4* __restrict__ rsrc,
                                                 const float* __restrict__ dsrc, int total, unsigned E1, unsigned E2,
                                                 bool v1, bool v2ok, const float4& ra, float dFX, int hbase,
                                                 v2 (&fh)[3], v2 (&fl)[3], int* hist) {
    constexpr int NB = SIMOX_NRDF + 2;
    const PackTab& T = Q.tab[TI];
    const float kcqa = Q.kc * ra.w;
    const float kcqaZY = T.kcZY * ra.w;
    const float4 t1 = etab[(E1 >> kSkinCodeShift) & kCodeMask];
    const float4 t2 = etab[(E2 >> kSkinCodeShift) & kCodeMask];
    int i1 = (int)(E1 & kIdxMask) + __float_as_int(t1.w);
    int i2 = (int)(E2 & kIdxMask) + __float_as_int(t2.w);
    if (TILED) {   // keep every shared load inside the tile
        i1 = (unsigned)i1 < (unsigned)total ? i1 : 0;
        i2 = (unsigned)i2 < (unsigned)total ? i2 : 0;
    }
    const float4 B1 = rsrc[i1], B2 = rsrc[i2];
    const float D1 = dsrc[i1], D2 = dsrc[i2];
    const v2 dx = mk2((ra.x - B1.x) - t1.x, (ra.x - B2.x) - t2.x);
    const v2 dy = mk2((ra.y - B1.y) - t1.y, (ra.y - B2.y) - t2.y);
    const v2 dz = mk2((ra.z - B1.z) - t1.z, (ra.z - B2.z) - t2.z);
    const v2 r2 = fma2(dx, dx, fma2(dy, dy, dz * dz));
    v2 fs = pair_fs_pk<SAME, MHOMO>(T, Q, r2, mk2(B1.w, B2.w), mk2(D1, D2), dFX, kcqa, kcqaZY);
    // slots past the end of a group evaluated a placeholder pair: drop it
    fs = mk2(v1 ? fs.v.x : 0.f, v2ok ? fs.v.y : 0.f);
    two_sum2(fh[0], fl[0], fs * dx);
    two_sum2(fh[1], fl[1], fs * dy);
    two_sum2(fh[2], fl[2], fs * dz);
    if (RDF) {
        // INT(r/dr) of the pair's FP32 distance, counted once, by the reference's i
        if (E1 & kIsA) {
            const float r = r2.v.x * rsqrt_approx(r2.v.x);
            atomicAdd(&hist[hbase + min(max((int)(r * Q.inv_dr), 0), NB - 1)], 2);
        }
        if (E2 & kIsA) {
            const float r = r2.v.y * rsqrt_approx(r2.v.y);
            atomicAdd(&hist[hbase + min(max((int)(r * Q.inv_dr), 0), NB - 1)], 2);
        }
    }
}

// The atoms [b0, b1) of one CTA, one warp per atom (taken from a shared
// counter), two row entries per lane per batch, the next batch's entries
// loaded before this batch's arithmetic.
template <bool RDF, bool TILED>
__device__ __forceinline__ void force_tile_atoms(const PackParams& Q, const float4* etab, const float4* __restrict__ rsrc,
                                                 const float* __restrict__ dsrc, int total, int b0, int b1, int* next,
                                                 const float4* __restrict__ frec, const int* __restrict__ ts,
                                                 const int2* __restrict__ nn, const unsigned* __restrict__ nbr,
                                                 const float* __restrict__ dF_f, const int* __restrict__ sorted, int g0,
                                                 double* __restrict__ f, int* hist, int& bad) {
    constexpr int NB = SIMOX_NRDF + 2;
    const int lane = threadIdx.x & 31;
    const int cap = Q.cap;
    for (;;) {
        int X = 0;
        if (lane == 0) X = atomicAdd(next, 1);
        X = __shfl_sync(0xffffffffu, X, 0) + b0;
        if (X >= b1) break;
        const float4 ra = frec[X];
        const int sX = ts[X];
        const float dFX = dF_f[X];
        const int2 m = nn[X];
        const unsigned* row = nbr + (size_t)X * cap;
        v2 fh[3] = {bc(0.f), bc(0.f), bc(0.f)}, fl[3] = {bc(0.f), bc(0.f), bc(0.f)};
        const bool metal = sX == g0;
        if (!metal && sX != 3) {
            if (m.x + m.y > 0) bad |= ST_UNKNOWN_PAIR;
        } else {
            // one stream of 64-entry batches over both groups: metal partners
            // (row[k]) then oxygen partners (row[cap - 1 - k])
            const int nb0 = (m.x + 63) >> 6, nb = nb0 + ((m.y + 63) >> 6);
            const unsigned pad = ((unsigned)kSelfEntry << kSkinCodeShift) | (unsigned)X;   // an in-tile placeholder
            auto load = [&](int j, unsigned& a, unsigned& b) {
                const bool g1 = j >= nb0;
                const int kb = (g1 ? j - nb0 : j) << 6, mg = g1 ? m.y : m.x;
                const unsigned* p = g1 ? row + (cap - 1 - kb - lane) : row + kb + lane;
                const int dir = g1 ? -32 : 32;
                a = kb + lane < mg ? p[0] : pad;
                b = kb + 32 + lane < mg ? p[dir] : pad;
            };
            unsigned na = pad, nbE = pad;
            if (nb > 0) load(0, na, nbE);
            for (int j = 0; j < nb; j++) {
                const unsigned E1 = na, E2 = nbE;
                if (j + 1 < nb) load(j + 1, na, nbE);
                const bool g1 = j >= nb0;
                const int kb = (g1 ? j - nb0 : j) << 6, mg = g1 ? m.y : m.x;
                const bool v1 = kb + lane < mg, v2ok = kb + 32 + lane < mg;
                const int hb = ((metal ? 0 : 2) + (g1 ? 1 : 0)) * NB;
                if (metal) {
                    if (!g1) force_batch_tile<true, true, RDF, TILED, 0>(Q, etab, rsrc, dsrc, total, E1, E2, v1, v2ok, ra, dFX, hb, fh, fl, hist);
                    else force_batch_tile<false, false, RDF, TILED, 1>(Q, etab, rsrc, dsrc, total, E1, E2, v1, v2ok, ra, dFX, hb, fh, fl, hist);
                } else {
                    if (!g1) force_batch_tile<false, false, RDF, TILED, 2>(Q, etab, rsrc, dsrc, total, E1, E2, v1, v2ok, ra, dFX, hb, fh, fl, hist);
                    else force_batch_tile<true, false, RDF, TILED, 3>(Q, etab, rsrc, dsrc, total, E1, E2, v1, v2ok, ra, dFX, hb, fh, fl, hist);
                }
            }
        }
        double fx = ((double)fh[0].v.x + (double)fl[0].v.x) + ((double)fh[0].v.y + (double)fl[0].v.y);
        double fy = ((double)fh[1].v.x + (double)fl[1].v.x) + ((double)fh[1].v.y + (double)fl[1].v.y);
        double fz = ((double)fh[2].v.x + (double)fl[2].v.x) + ((double)fh[2].v.y + (double)fl[2].v.y);
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
}

template <bool RDF>
__global__ void __launch_bounds__(kTileThreads, kTileBlocks)
    force_tile_kernel(const __grid_constant__ PackParams Q, int splits, const int* __restrict__ cs_start,
                      const int* __restrict__ cs_entries, const float4* __restrict__ frec,
                      const int* __restrict__ ts, const int2* __restrict__ nn, const unsigned* __restrict__ nbr,
                      const float* __restrict__ dF_f, const int* __restrict__ sorted, int g0,
                      double* __restrict__ f, int* __restrict__ rdf, int* __restrict__ status) {
    extern __shared__ __align__(16) unsigned char tile_smem[];
    float4* trec = reinterpret_cast<float4*>(tile_smem);
    float* tdf = reinterpret_cast<float*>(trec + kTileCap);
    __shared__ float4 etab[kEntries];          // o_e * Lcs (x, y, z) and tile index delta (w)
    __shared__ int eoff[kEntries + 1], estart[kEntries];
    __shared__ int next;
    constexpr int NB = SIMOX_NRDF + 2;
    __shared__ int hist[RDF ? 4 * NB : 1];     // (metal, O) x (metal, O) partner kinds
    const int cell = blockIdx.x / splits, part = blockIdx.x - cell * splits;
    const int tid = threadIdx.x;
    if (tid < kEntries) {
        const int nc = cs_entries[cell * kEntries + tid];
        const int s0 = cs_start[nc];
        estart[tid] = s0;
        eoff[tid + 1] = cs_start[nc + 1] - s0;
    }
    if (tid == 0) {
        eoff[0] = 0;
        next = 0;
    }
    if (RDF)
        for (int k = tid; k < 4 * NB; k += kTileThreads) hist[k] = 0;
    __syncthreads();
    if (tid == 0)
        for (int e = 0; e < kEntries; e++) eoff[e + 1] += eoff[e];
    __syncthreads();
    const int total = eoff[kEntries];
    const bool tiled = total <= kTileCap;
    if (tid < kEntries) {
        const float4 o = Q.sh[tid];
        etab[tid] = make_float4(o.x, o.y, o.z, __int_as_float(tiled ? eoff[tid] - estart[tid] : 0));
    }
    if (tiled) {
        int e = 0;
        for (int i = tid; i < total; i += kTileThreads) {
            while (eoff[e + 1] <= i) e++;
            const int src = estart[e] + (i - eoff[e]);
            cp_async16(&trec[i], frec + src);
            cp_async4(&tdf[i], dF_f + src);
        }
        cp_async_commit();
        cp_async_wait<0>();
    }
    __syncthreads();
    const int a0 = cs_start[cell], na = cs_start[cell + 1] - a0;
    const int b0 = a0 + (int)((long long)na * part / splits);
    const int b1 = a0 + (int)((long long)na * (part + 1) / splits);
    int bad = 0;
    if (tiled)
        force_tile_atoms<RDF, true>(Q, etab, trec, tdf, total, b0, b1, &next, frec, ts, nn, nbr, dF_f, sorted, g0, f,
                                    hist, bad);
    else
        force_tile_atoms<RDF, false>(Q, etab, frec, dF_f, total, b0, b1, &next, frec, ts, nn, nbr, dF_f, sorted, g0,
                                     f, hist, bad);
    if (bad) atomicOr(status, bad);
    if (RDF) {
        __syncthreads();
        for (int k = tid; k < 4 * NB; k += kTileThreads) {
            const int v = hist[k];
            if (v) {
                const int pr = k / NB, bin = k - pr * NB;
                const int si = pr >= 2 ? 3 : g0, sj = (pr & 1) ? 3 : g0;
                atomicAdd(&rdf[si + 5 * sj + 25 * bin], v);
            }
        }
    }
}


// pass 2 -------------------------------------------------------------------
// Block shape: FP32 uses 256-thread CTAs, 3 per SM (<= 85 registers); the
// FP64 variant needs ~150 registers, so 128-thread CTAs pack 3 per SM.
template <typename R> struct ForceShape {
    static constexpr int threads = sizeof(R) == 4 ? 256 : 128;
    static constexpr int blocks = sizeof(R) == 4 ? 3 : 4;
};

template <typename R, bool EFLAG, bool RDF>
__global__ void __launch_bounds__(ForceShape<R>::threads, ForceShape<R>::blocks)
    force_kernel(PairParams P, const PairTab<R>* __restrict__ tab, const double4* __restrict__ xq,
                 const int* __restrict__ ts, const int2* __restrict__ nn, const unsigned* __restrict__ nbr,
                 const double* __restrict__ dF_s, const float* __restrict__ dF_f, const int* __restrict__ sorted,
                 double* __restrict__ f, double* __restrict__ acc, int* __restrict__ rdf, int* __restrict__ status) {
    constexpr int NT = ForceShape<R>::threads;
    __shared__ PairTab<R> st[kSpecies * kSpecies];
    __shared__ double red[NT / 32];
    constexpr int NB = SIMOX_NRDF + 2;
    __shared__ int hist[RDF ? kSpecies * kSpecies * NB : 1];
    for (int k = threadIdx.x; k < kSpecies * kSpecies; k += blockDim.x) st[k] = tab[k];
    if (RDF)
        for (int k = threadIdx.x; k < kSpecies * kSpecies * NB; k += blockDim.x) hist[k] = 0;
    __syncthreads();
    const int lane = threadIdx.x & 31;
    const int wpb = blockDim.x >> 5;
    double ep = 0.0, ed = 0.0, ec = 0.0;
    int bad = 0;
    for (int X = blockIdx.x * wpb + (threadIdx.x >> 5); X < P.n; X += gridDim.x * wpb) {
        const double4 xa = xq[X];
        const int sX = ts[X];
        const R qa = (R)xa.w;
        const R dFX = (R)dF_s[X];
        const int2 m = nn[X];
        const unsigned* row = nbr + (size_t)X * P.cap;
        double fx = 0.0, fy = 0.0, fz = 0.0;
        if (sX >= kSpecies) {
            if (m.x + m.y > 0) bad |= ST_UNKNOWN_PAIR;
        } else if (sizeof(R) == 8) {
            // FP64: one table-driven body over the whole row (the inlined FP64
            // exp/erfc sequences make per-species copies overflow the I-cache)
            force_group<R, false, false, EFLAG, RDF>(P, st, row, 2, m.x + m.y, lane, xa, sX, m.x, qa, dFX, xq, ts,
                                                     dF_s, dF_f, fx, fy, fz, ep, ed, ec, hist, bad);
        } else if (sX < 3) {   // metal X: metal partners (same species) then oxygen partners
            force_group<R, true, true, EFLAG, RDF>(P, st, row, 0, m.x, lane, xa, sX, -1, qa, dFX, xq, ts, dF_s, dF_f, fx,
                                                   fy, fz, ep, ed, ec, hist, bad);
            force_group<R, false, false, EFLAG, RDF>(P, st, row, 1, m.y, lane, xa, sX, 3, qa, dFX, xq, ts, dF_s, dF_f,
                                                     fx, fy, fz, ep, ed, ec, hist, bad);
        } else {               // oxygen X: metal partners then oxygen partners
            force_group<R, false, false, EFLAG, RDF>(P, st, row, 0, m.x, lane, xa, sX, -1, qa, dFX, xq, ts, dF_s, dF_f,
                                                     fx, fy, fz, ep, ed, ec, hist, bad);
            force_group<R, true, false, EFLAG, RDF>(P, st, row, 1, m.y, lane, xa, sX, 3, qa, dFX, xq, ts, dF_s, dF_f, fx,
                                                    fy, fz, ep, ed, ec, hist, bad);
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
        block_add<NT>(0.5 * ep, acc, A_EPAIR, red);
        block_add<NT>(0.5 * ed, acc, A_EDIR, red);
        block_add<NT>(0.5 * ec, acc, A_ECTIP, red);
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

// FP64 energies of the mixed-precision mode (force.f90:84-98, 101-140, 256-351).
// Per atom X (one warp) the FP64 density rho_X is summed over the whole exact
// row and gives the embedding energy F(rho_X); the pair energies (phi, Ewald
// real space, CTIP) are evaluated once per pair, on the side of the
// reference's i (list bit 31).  Those entries are queued per warp in shared
// memory and evaluated 32 at a time, so the FP64 exponentials run on full
// warps.  Six CTAs per SM (80 registers, 24 warps) hide the partner gathers
// better than the unconstrained 92 registers (20 warps): 1.23 against 1.48 ms
// at 128k corundum.
constexpr int EN_THREADS = 128;


struct EnQueue {
    double r[64];
    double qb[64];
    int t[64];
};

__global__ void __launch_bounds__(EN_THREADS, 6)
    energy_kernel(PairParams P, const PairTab<double>* __restrict__ tab, const double4* __restrict__ xq,
                  const int* __restrict__ ts, const int2* __restrict__ nn, const unsigned* __restrict__ nbr,
                  EmbedParams E, double* __restrict__ acc, int* __restrict__ status) {
    __shared__ PairTab<double> st[kSpecies * kSpecies];
    __shared__ EnQueue qu[EN_THREADS / 32];
    __shared__ double red[EN_THREADS / 32];
    for (int k = threadIdx.x; k < kSpecies * kSpecies; k += blockDim.x) st[k] = tab[k];
    __syncthreads();
    const int lane = threadIdx.x & 31, wpb = blockDim.x >> 5;
    EnQueue& Qw = qu[threadIdx.x >> 5];
    const unsigned lt = (1u << lane) - 1u;
    double ep = 0.0, ed = 0.0, ec = 0.0, eg = 0.0;
    int bad = 0;
    for (int X = blockIdx.x * wpb + (threadIdx.x >> 5); X < P.n; X += gridDim.x * wpb) {
        const double4 xa = xq[X];
        const int sX = ts[X];
        const int2 m = nn[X];
        const int mt = m.x + m.y;
        const unsigned* row = nbr + (size_t)X * P.cap;
        double rho = 0.0;
        int qn = 0;   // queued pairs (warp-uniform)
        if (sX < kSpecies) {
            for (int base = 0; base < mt; base += 32) {
                const int k = base + lane;
                bool isa = false;
                double r = 0.0, qb = 0.0;
                int t = 0;
                if (k < mt) {
                    const unsigned ent = row[row_slot(2, k, P.cap, m.x)];
                    const int Y = (int)(ent & kIdxMask);
                    const int sY = ts[Y];
                    if (sY < kSpecies) {
                        const double4 xb = xq[Y];
                        double dx, dy, dz;
                        min_image(xa, xb, P, dx, dy, dz);
                        r = sqrt(__dadd_rn(__dadd_rn(__dmul_rn(dx, dx), __dmul_rn(dy, dy)), __dmul_rn(dz, dz)));
                        t = sX * kSpecies + sY;
                        const PairTab<double>& T = st[t];
                        rho += T.d_fe * zhou_val<double>(r, T.d_inv_re, T.d_c, T.d_lam);   // force.f90:84
                        isa = (ent & kIsA) != 0u;
                        qb = xb.w;
                    } else {
                        bad |= ST_UNKNOWN_PAIR;
                    }
                }
                const unsigned mk = __ballot_sync(0xffffffffu, isa);
                if (isa) {
                    const int pos = qn + __popc(mk & lt);
                    Qw.r[pos] = r;
                    Qw.qb[pos] = qb;
                    Qw.t[pos] = t;
                }
                qn += __popc(mk);
                __syncwarp();
                if (qn >= 32) {   // a full warp of pair energies
                    const double rr = Qw.r[lane], qq = Qw.qb[lane];
                    const int tt = Qw.t[lane];
                    __syncwarp();
                    if (lane < qn - 32) {
                        Qw.r[lane] = Qw.r[lane + 32];
                        Qw.qb[lane] = Qw.qb[lane + 32];
                        Qw.t[lane] = Qw.t[lane + 32];
                    }
                    qn -= 32;
                    __syncwarp();
                    pair_energy_fp64(st[tt], rr, 1.0 / rr, xa.w, qq, P.a, ep, ed, ec);
                }
            }
            if (lane < qn) pair_energy_fp64(st[Qw.t[lane]], Qw.r[lane], 1.0 / Qw.r[lane], xa.w, Qw.qb[lane], P.a, ep, ed, ec);
            __syncwarp();
        } else if (mt > 0) {
            bad |= ST_UNKNOWN_PAIR;
        }
        rho = warp_sum(rho);
        if (lane == 0) {
            double F, dF;
            if (embed(E, sX, rho, F, dF)) bad |= ST_UNKNOWN_ELEMENT;
            eg += F;
        }
    }
    if (bad) atomicOr(status, bad);
    block_add<EN_THREADS>(ep, acc, A_EPAIR, red);
    block_add<EN_THREADS>(ed, acc, A_EDIR, red);
    block_add<EN_THREADS>(ec, acc, A_ECTIP, red);
    block_add<EN_THREADS>(eg, acc, A_EGROUP, red);
}


// Forces use the context's precision.  Energies are FP64 in both modes: the
// FP64 context evaluates them inside its force pass, the mixed context with
// the separate FP64 energy pass (energy_kernel) after its mixed force pass.
static bool use_fp64(const simox_ctx* c, bool) { return c->precision == SIMOX_FP64; }

int eam_density(simox_ctx* c, bool eflag) {
    int st = ensure_list(c);
    if (st) return st;
    if (c->n == 0) return SIMOX_OK;
    PairParams P = pair_params(c);
    EmbedParams E = embed_params(c->pot);
    // a half list carries each pair once: its densities come only from the
    // half-list filter pass (both atoms of each pair)
    if (!c->rho_ready && half_path(c)) {
        memset_async(c, c->nn_max, 0, sizeof(int), c->stream);
        memset_async(c, c->nn_tot, 0, sizeof(unsigned long long), c->stream);
        if ((st = filter_density(c))) return st;
    }
    // the skin filter already produced rho and F' in the context's precision
    if (c->rho_ready) {
        if (eflag && c->precision == SIMOX_FP64) {
            Launch L(c, "eam_embed_energy");
            embed_energy_kernel<<<(c->n + 255) / 256, 256, 0, c->stream>>>(c->n, c->t_s, c->rho_s, E, c->acc);
        }
        c->eam_valid = true;
        return check_launch(c);
    }
    Launch L(c, use_fp64(c, eflag) ? "eam_density_fp64" : "eam_density");
    if (!use_fp64(c, eflag))
        density_kernel<float><<<pair_grid(c), PK_THREADS, 0, c->stream>>>(P, c->tab_f, c->xq_s, c->t_s,
                                                                         reinterpret_cast<const int2*>(c->nn), c->nbr, E,
                                                                         c->rho_s, c->dF_s, c->dF_f, c->acc, c->status, 0);
    else
        density_kernel<double><<<pair_grid(c), PK_THREADS, 0, c->stream>>>(P, c->tab_d, c->xq_s, c->t_s,
                                                                          reinterpret_cast<const int2*>(c->nn), c->nbr,
                                                                          E, c->rho_s, c->dF_s, c->dF_f, c->acc,
                                                                          c->status, eflag);
    c->eam_valid = true;
    c->rho_ready = false;   // rho/F' now in the precision of this pass
    return check_launch(c);
}


int filter_density(simox_ctx* c) {
    if (half_path(c)) {
        if (int st = filter_density_half(c)) return st;
        c->rho_ready = true;
        return SIMOX_OK;
    }
    FilterParams F;
    F.pp = pair_params(c);
    F.rcut2 = c->rcut2;
    F.rcut2f = (float)c->rcut2;
    F.band = filter_band(c);
    F.nc = make_int3(c->nc[0], c->nc[1], c->nc[2]);
    F.cap_s = c->cap_s;
    stencil_shifts(c, F.sh);
    EmbedParams E = embed_params(c->pot);
    if (c->n > 0) {
        Launch L(c, "neighbor_filter_density");
        const int g = std::min((c->n + 7) / 8, num_sms(c) * 8);
        if (c->precision == SIMOX_FP64)
            filter_density_kernel<double><<<g, 256, 0, c->stream>>>(
                F, c->tab_d, c->xq_s, c->rec_s, c->pair_order, reinterpret_cast<const int2*>(c->nn_s), c->nbr_s,
                reinterpret_cast<int2*>(c->nn), c->nbr, E, c->rho_s, c->dF_s, c->dF_f, c->status, c->nn_max, c->nn_tot,
                c->g0_species);
        else
            filter_density_kernel<float><<<g, 256, 0, c->stream>>>(
                F, c->tab_f, c->xq_s, c->rec_s, c->pair_order, reinterpret_cast<const int2*>(c->nn_s), c->nbr_s,
                reinterpret_cast<int2*>(c->nn), c->nbr, E, c->rho_s, c->dF_s, c->dF_f, c->status, c->nn_max, c->nn_tot,
                c->g0_species);
    }
    int st = check_launch(c);
    if (st) return st;
    c->rho_ready = true;
    return SIMOX_OK;
}

template <typename R>
static void launch_force(simox_ctx* c, const PairTab<R>* tab, bool eflag, bool rdf) {
    PairParams P = pair_params(c);
    constexpr int PK_THREADS = ForceShape<R>::threads;
    const int wpb = PK_THREADS / 32;
    int g = std::min((c->n + wpb - 1) / wpb, num_sms(c) * 3 * (256 / PK_THREADS) * 2);
    if (g < 1) g = 1;
    if (eflag && rdf)
        force_kernel<R, true, true><<<g, PK_THREADS, 0, c->stream>>>(P, tab, c->xq_s, c->t_s, reinterpret_cast<const int2*>(c->nn), c->nbr, c->dF_s, c->dF_f,
                                                                     c->pair_order, c->f, c->acc, c->rdf, c->status);
    else if (eflag)
        force_kernel<R, true, false><<<g, PK_THREADS, 0, c->stream>>>(P, tab, c->xq_s, c->t_s, reinterpret_cast<const int2*>(c->nn), c->nbr, c->dF_s, c->dF_f,
                                                                      c->pair_order, c->f, c->acc, c->rdf, c->status);
    else if (rdf)
        force_kernel<R, false, true><<<g, PK_THREADS, 0, c->stream>>>(P, tab, c->xq_s, c->t_s, reinterpret_cast<const int2*>(c->nn), c->nbr, c->dF_s, c->dF_f,
                                                                      c->pair_order, c->f, c->acc, c->rdf, c->status);
    else
        force_kernel<R, false, false><<<g, PK_THREADS, 0, c->stream>>>(P, tab, c->xq_s, c->t_s, reinterpret_cast<const int2*>(c->nn), c->nbr, c->dF_s, c->dF_f,
                                                                       c->pair_order, c->f, c->acc, c->rdf, c->status);
}

static constexpr size_t kTileSmem = (size_t)kTileCap * (sizeof(float4) + sizeof(float));

// dynamic shared memory of the tiled force pass, once per device
static int tile_prepare(int device) {
    static std::atomic<bool> done[64] = {};   // contexts may run on several host threads
    if (device >= 0 && device < 64 && done[device].load()) return SIMOX_OK;
    const int b = (int)kTileSmem;
    cudaError_t e1 = cudaFuncSetAttribute(force_tile_kernel<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, b);
    cudaError_t e2 = cudaFuncSetAttribute(force_tile_kernel<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, b);
    cudaError_t e3 = cudaFuncSetAttribute(force_tile_kernel<true>, cudaFuncAttributePreferredSharedMemoryCarveout,
                                          cudaSharedmemCarveoutMaxShared);
    cudaError_t e4 = cudaFuncSetAttribute(force_tile_kernel<false>, cudaFuncAttributePreferredSharedMemoryCarveout,
                                          cudaSharedmemCarveoutMaxShared);
    if (e1 != cudaSuccess || e2 != cudaSuccess || e3 != cudaSuccess || e4 != cudaSuccess) return SIMOX_E_CUDA;
    if (device >= 0 && device < 64) done[device] = true;
    return SIMOX_OK;
}

static int energy_pass(simox_ctx* c) {
    if (half_path(c)) return energy_half(c);
    Launch L(c, "pair_energy_fp64");
    const int wpb = EN_THREADS / 32;
    const int g = std::max(1, std::min((c->n + wpb - 1) / wpb, num_sms(c) * 12));
    energy_kernel<<<g, EN_THREADS, 0, c->stream>>>(pair_params(c), c->tab_d, c->xq_s, c->t_s,
                                                  reinterpret_cast<const int2*>(c->nn), c->nbr, embed_params(c->pot),
                                                  c->acc, c->status);
    return check_launch(c);
}

static int mixed_forces(simox_ctx* c, bool rdf);

int pair_forces(simox_ctx* c, bool eflag, bool rdf) {
    if (!c->eam_valid) return SIMOX_E_STATE;
    if (c->n == 0) return SIMOX_OK;
    if (c->precision != SIMOX_FP64) {
        if (int st = mixed_forces(c, rdf)) return st;
        return eflag ? energy_pass(c) : SIMOX_OK;
    }
    Launch L(c, eflag ? "pair_force_fp64_energy" : "pair_force_fp64");
    launch_force<double>(c, c->tab_d, eflag, rdf);
    return check_launch(c);
}

static int mixed_forces(simox_ctx* c, bool rdf) {
    if (half_path(c)) return force_half(c, rdf);
    const bool eflag = false;
    if (!use_fp64(c, eflag) && c->using_skin && c->g0_species >= 0) {
        Launch L(c, "pair_force");
        PairParams P = pair_params(c);
        if (int st = tile_prepare(c->device)) return st;
        PackParams Q;
        std::memset(&Q, 0, sizeof(Q));
        Q.pa = (float)(kErfcP * P.a);
        Q.na2l = (float)(-P.a * P.a * 1.4426950408889634);
        Q.tas = (float)(2.0 * P.a / SX_SQRTPI);
        Q.kc = (float)P.kc;
        Q.inv_dr = (float)(1.0 / P.dr_rdf);
        Q.cap = P.cap;
        stencil_shifts(c, Q.sh);
        const int g0 = c->g0_species;
        Q.tab[0] = pack_tab(c->pot, g0, g0);
        Q.tab[1] = pack_tab(c->pot, g0, 3);
        Q.tab[2] = pack_tab(c->pot, 3, g0);
        Q.tab[3] = pack_tab(c->pot, 3, 3);
        const int splits = std::max(1, std::min(16, c->force_splits));
        const int g = c->ncell_s * splits;
        const int2* nn = reinterpret_cast<const int2*>(c->nn);
        if (rdf)
            force_tile_kernel<true><<<g, kTileThreads, kTileSmem, c->stream>>>(
                Q, splits, c->cs_start, c->cs_entries, c->frec_s, c->t_s, nn, c->nbr, c->dF_f, c->pair_order, g0,
                c->f, c->rdf, c->status);
        else
            force_tile_kernel<false><<<g, kTileThreads, kTileSmem, c->stream>>>(
                Q, splits, c->cs_start, c->cs_entries, c->frec_s, c->t_s, nn, c->nbr, c->dF_f, c->pair_order, g0,
                c->f, c->rdf, c->status);
        return check_launch(c);
    }
    Launch L(c, "pair_force");
    launch_force<float>(c, c->tab_f, eflag, rdf);
    return check_launch(c);
}

}  // namespace sx
