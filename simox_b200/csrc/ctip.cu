// ctip.cu -- CTIP_SOLVER (ctip.f90:3-212), matrix-free.
//
// The reference minimises U(q) = chi.q + 1/2 q.A q + Z-terms + penalty(q) by a
// nonlinear CG: g = -dU/dq (dUdq, ctip.f90:307-333), beta = sum(g)/sum(g_old),
// d = g + beta p, p = d - mean(d), alpha = root of h(b) = -sum g(q+bp).p on
// [-1,1] (BRENT_SOLVER, ctip.f90:216-304), q += alpha p, stop when
// MAXVAL(|p|)*|alpha| <= 1e-3.  It stores the short-range matrices (N x 500)
// and re-evaluates the PME potential 3 + n_Brent times per iteration.
//
// Here A p is formed once per iteration without stored matrices: the pair
// kernel recomputes sym_ij = kc(fifj + erfc(a r)/r) from the neighbour list
// and the PME potential of p comes from pme_potential().  Because U is
// quadratic apart from the per-atom penalty 2w(min(0,q-qmin)+max(0,q-qmax)),
//   g(q + b p) = g(q) - b A p - [pen'(q + b p) - pen'(q)],
// so h(b) = -g.p + b p.Ap + sum_i p_i [pen'_i(q_i + b p_i) - pen'_i(q_i)] is
// exact and piecewise linear, and costs one reduction over the atoms whose
// charge can cross a bound for b in [-1,1].  The reference's Brent iteration
// (same bracket, tolerances 1e-8 / 1e-11, 100-step limit) runs on it inside
// one CTA, so each CG step takes the reference's alpha up to the rounding of
// h.  g is then updated in place (the reference recomputes it from scratch;
// the two agree in exact arithmetic).  Vectors, dots and reductions are FP64.
#include "simox_internal.cuh"

#include <algorithm>
#include <cmath>
#include <cstring>

namespace sx {

constexpr int CT_THREADS = 256;

// scalar slots in c->line
enum : int { L_GSUM_OLD = 0, L_ALPHA, L_ERROR, L_DONE, L_NEVAL, L_ITERS, L_CHUNK, L_END };

struct CtipParams {
    double3 box, ibox;
    double a, kc;
    int cap, n;
};

template <typename R> __device__ __forceinline__ R cexp(R x);
template <> __device__ __forceinline__ double cexp<double>(double x) { return exp(x); }
template <> __device__ __forceinline__ float cexp<float>(float x) { return __expf(x); }
template <typename R> __device__ __forceinline__ R cerfc(R x);
template <> __device__ __forceinline__ double cerfc<double>(double x) { return erfc(x); }
// Numerical Recipes "erfcc" (Chebyshev fit, fractional error < 1.2e-7, x >= 0)
template <> __device__ __forceinline__ float cerfc<float>(float z) {
    const float t = __fdividef(1.0f, 1.0f + 0.5f * z);
    const float p = -1.26551223f + t * (1.00002368f + t * (0.37409196f + t * (0.09678418f +
                    t * (-0.18628806f + t * (0.27886807f + t * (-1.13520398f + t * (1.48851587f +
                    t * (-0.82215223f + t * 0.17087277f))))))));
    return t * __expf(p - z * z);
}

__device__ __forceinline__ double pen_d(double q, double lo, double hi) {
    // 2w*(dqmin + dqmax) with dqmin = min(0, q-qmin), dqmax = max(0, q-qmax)  ctip.f90:317-322
    double a = q - lo, b = q - hi;
    if (a >= 0.0) a = 0.0;
    if (b <= 0.0) b = 0.0;
    return 2.0 * SX_WPEN * (a + b);
}

// One group of X's row: sr += sum_Y sym_XY v_Y; cz += sum_Y Z_Y asym_XY.
// SAME: the partner has X's species (one Slater exponential).
template <typename R, bool WITH_C, bool SAME>
__device__ __forceinline__ void ctip_group(const CtipParams& P, const PairTab<R>* st, const unsigned* row, int g,
                                           int mg, int lane, const double4& xa, int sX, int sY_fixed,
                                           const double4* __restrict__ xq, const int* __restrict__ ts,
                                           const double* __restrict__ vin, double& sr, double& cz) {
    const R a = (R)P.a, kc = (R)P.kc;
    const int nm = g == 2 ? sY_fixed : 0;   // group 2: the whole row, sY_fixed = number of metal partners
    if (g == 2) sY_fixed = -1;
    for (int k = lane; k < mg; k += 32) {
        const int slot = g == 0 ? k : (g == 1 ? P.cap - 1 - k : (k < nm ? k : P.cap - 1 - (k - nm)));
        const int Y = (int)(row[slot] & kIdxMask);
        const double4 xb = xq[Y];
        const int sY = sY_fixed >= 0 ? sY_fixed : ts[Y];
        if (sY >= kSpecies || (SAME && sY != sX)) continue;   // flagged by the force pass
        double dx = __dsub_rn(xa.x, xb.x), dy = __dsub_rn(xa.y, xb.y), dz = __dsub_rn(xa.z, xb.z);
        dx = __dsub_rn(dx, __dmul_rn(P.box.x, rint(dx * P.ibox.x)));
        dy = __dsub_rn(dy, __dmul_rn(P.box.y, rint(dy * P.ibox.y)));
        dz = __dsub_rn(dz, __dmul_rn(P.box.z, rint(dz * P.ibox.z)));
        const double r2d = __dadd_rn(__dadd_rn(__dmul_rn(dx, dx), __dmul_rn(dy, dy)), __dmul_rn(dz, dz));
        R r, ir;
        if (sizeof(R) == 8) { r = (R)sqrt(r2d); ir = R(1) / r; }
        else { ir = (R)rsqrtf((float)r2d); r = (R)r2d * ir; }
        const PairTab<R>& T = st[sX * kSpecies + sY];
        const R eX = cexp<R>(R(-2) * T.xi_x * r);
        // fifj (ctip.f90:91-100) = -(eX SX(r) + eY SY(r))/r
        R num = eX * (T.Sx[0] + r * (T.Sx[1] + r * (T.Sx[2] + r * T.Sx[3])));
        if (!SAME) num += cexp<R>(R(-2) * T.xi_y * r) * (T.Sy[0] + r * T.Sy[1]);
        const R fifj = -num * ir;
        const R sym = kc * (fifj + cerfc<R>(a * r) * ir);            // ctip.f90:108
        sr += (double)sym * vin[Y];
        if (WITH_C) {
            const R afbX = -eX * (T.xi_x + ir);                         // ctip.f90:86,96
            cz += (double)(T.Z_y * kc * (afbX - fifj));                 // ctip.f90:106 x XJZ(j,3)
        }
    }
}

// Pair pass over the list: out[X] = sum_Y sym_XY v_Y ; optional cconst[X] = chi_X + sum_Y Z_Y asym_XY
template <typename R, bool WITH_C>
__global__ void __launch_bounds__(CT_THREADS)
    ctip_pair_kernel(CtipParams P, const PairTab<R>* __restrict__ tab, const double4* __restrict__ xq,
                     const int* __restrict__ ts, const int2* __restrict__ nn, const unsigned* __restrict__ nbr,
                     const double* __restrict__ vin, double* __restrict__ out, double* __restrict__ cconst,
                     CtipSpecies S) {
    __shared__ PairTab<R> st[kSpecies * kSpecies];
    for (int k = threadIdx.x; k < kSpecies * kSpecies; k += blockDim.x) st[k] = tab[k];
    __syncthreads();
    const int lane = threadIdx.x & 31, wpb = blockDim.x >> 5;
    for (int X = blockIdx.x * wpb + (threadIdx.x >> 5); X < P.n; X += gridDim.x * wpb) {
        const double4 xa = xq[X];
        const int sX = ts[X];
        const int2 m = nn[X];
        const unsigned* row = nbr + (size_t)X * P.cap;
        double sr = 0.0, cz = 0.0;
        if (sX >= kSpecies) {
        } else if (sizeof(R) == 8) {   // FP64: one table-driven body (I-cache)
            ctip_group<R, WITH_C, false>(P, st, row, 2, m.x + m.y, lane, xa, sX, m.x, xq, ts, vin, sr, cz);
        } else if (sX < 3) {
            ctip_group<R, WITH_C, true>(P, st, row, 0, m.x, lane, xa, sX, -1, xq, ts, vin, sr, cz);
            ctip_group<R, WITH_C, false>(P, st, row, 1, m.y, lane, xa, sX, 3, xq, ts, vin, sr, cz);
        } else {
            ctip_group<R, WITH_C, false>(P, st, row, 0, m.x, lane, xa, sX, -1, xq, ts, vin, sr, cz);
            ctip_group<R, WITH_C, true>(P, st, row, 1, m.y, lane, xa, sX, 3, xq, ts, vin, sr, cz);
        }
        sr = warp_sum(sr);
        if (WITH_C) cz = warp_sum(cz);
        if (lane == 0) {
            out[X] = sr;
            if (WITH_C) cconst[X] = S.chi[min(sX, 4)] + cz;
        }
    }
}

// g = -(c + J'q + phi + pen'(q) + sr)  with phi already in g (from pme_potential)
__global__ void __launch_bounds__(CT_THREADS)
    ctip_init_g_kernel(int n, const int* __restrict__ ts, const double* __restrict__ q,
                       const double* __restrict__ cc, const double* __restrict__ sr, double* __restrict__ g,
                       double* __restrict__ pv, CtipSpecies S, double* __restrict__ acc) {
    __shared__ double red[CT_THREADS / 32];
    double gs = 0.0;
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) {
        const int s = min(ts[i], 4);
        const double qi = q[i];
        const double v = -(cc[i] + S.Jp[s] * qi + g[i] + pen_d(qi, S.qmin[s], S.qmax[s]) + sr[i]);
        g[i] = v;
        pv[i] = 0.0;
        gs = v;
    }
    block_add<CT_THREADS>(gs, acc, A_GSUM, red);
}

// d = g + p*gsum/gsum_old (in pv); sum d   (ctip.f90:172-180)
__global__ void __launch_bounds__(CT_THREADS)
    ctip_dir_kernel(int n, const double* __restrict__ g, double* __restrict__ pv, const double* __restrict__ line,
                    double* __restrict__ acc) {
    __shared__ double red[CT_THREADS / 32];
    const double gsum = acc[A_GSUM], gold = line[L_GSUM_OLD];
    double ds = 0.0;
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) {
        const double d = g[i] + pv[i] * gsum / gold;
        pv[i] = d;
        ds = d;
    }
    block_add<CT_THREADS>(ds, acc, A_PSUM, red);
}

// p = d - sum(d)/N; max|p|   (ctip.f90:180-181, 187)
__global__ void ctip_proj_kernel(int n, double* __restrict__ pv, double* __restrict__ acc) {
    const double dm = acc[A_PSUM] / (double)n;
    double mx = 0.0;
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) {
        const double p = pv[i] - dm;
        pv[i] = p;
        mx = fabs(p);
    }
    mx = warp_max(mx);
    if ((threadIdx.x & 31) == 0 && mx > 0.0)
        atomicMax(reinterpret_cast<unsigned long long*>(acc + A_PMAX), (unsigned long long)__double_as_longlong(mx));
}

// Ap = phi(p) [already in Ap] + J' p + SR(p); dots g.p, p.Ap; active atoms
__global__ void __launch_bounds__(CT_THREADS)
    ctip_matvec_finish_kernel(int n, const int* __restrict__ ts, const double* __restrict__ q,
                              const double* __restrict__ g, const double* __restrict__ pv,
                              const double* __restrict__ sr, double* __restrict__ Ap, CtipSpecies S,
                              int* __restrict__ act, int* __restrict__ nact, double* __restrict__ acc) {
    __shared__ double red[CT_THREADS / 32];
    double gp = 0.0, pap = 0.0;
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) {
        const int s = min(ts[i], 4);
        const double p = pv[i];
        const double ap = Ap[i] + S.Jp[s] * p + sr[i];
        Ap[i] = ap;
        gp = g[i] * p;
        pap = p * ap;
        const double qi = q[i], ap_ = fabs(p);
        if (qi - ap_ < S.qmin[s] || qi + ap_ > S.qmax[s]) {
            int slot = atomicAdd(nact, 1);
            act[slot] = i;
        }
    }
    block_add<CT_THREADS>(gp, acc, A_GP, red);
    block_add<CT_THREADS>(pap, acc, A_PAP, red);
}

// BRENT_SOLVER (ctip.f90:216-304) replayed on the device.  h(b) is the
// exact closed form above; one CTA evaluates its penalty part over the
// active atoms per Brent step, and every thread runs the same Brent control
// flow on the same values, so the iterates (and the returned b) are the
// reference's up to the rounding of h.
__global__ void __launch_bounds__(1024)
    ctip_brent_kernel(const int* __restrict__ ts, const double* __restrict__ q, const double* __restrict__ pv,
                      const int* __restrict__ act, const int* __restrict__ nact, CtipSpecies S,
                      double* __restrict__ line, double* __restrict__ acc, double ecrit, int* __restrict__ status) {
    __shared__ double red[32];
    __shared__ double res;
    const double gp = acc[A_GP], pap = acc[A_PAP];
    const int na = *nact;
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, nw = blockDim.x >> 5;
    auto H = [&](double b) -> double {
        double s = 0.0;
        for (int k = threadIdx.x; k < na; k += blockDim.x) {
            const int i = act[k];
            const int sp = min(ts[i], 4);
            const double qi = q[i], p = pv[i];
            s += p * (pen_d(qi + b * p, S.qmin[sp], S.qmax[sp]) - pen_d(qi, S.qmin[sp], S.qmax[sp]));
        }
        s = warp_sum(s);
        if (lane == 0) red[w] = s;
        __syncthreads();
        if (w == 0) {
            double t = lane < nw ? red[lane] : 0.0;
            t = warp_sum(t);
            if (lane == 0) res = t;
        }
        __syncthreads();
        const double h = -gp + b * pap + res;   // = -sum g(q + b p) p
        __syncthreads();
        return h;
    };
    const double E_crit = 1.0e-8, E_end = 1.0e-11;
    double a = -1.0, b = 1.0, c, d = 0.0, e = 0.0, fa, fb, fc, xm, sv, x, y, z;
    fa = H(a);
    fb = H(b);
    c = b;
    fc = fb;
    double alpha = b;
    int n, ok = 0;
    for (n = 1; n <= 100; n++) {
        if ((fb > 0.0 && fc > 0.0) || (fb < 0.0 && fc < 0.0)) { c = a; fc = fa; d = b - a; e = d; }
        if (fabs(fc) < fabs(fb)) { a = b; b = c; c = a; fa = fb; fb = fc; fc = fa; }
        xm = 0.5 * (c - b);
        if (fabs(xm) < E_crit || fabs(fb) < E_end) { alpha = b; ok = 1; break; }
        if (fabs(e) >= E_crit && fabs(fa) > fabs(fb)) {
            sv = fb / fa;
            if (a == c) { x = 2.0 * xm * sv; y = 1.0 - sv; }
            else {
                y = fa / fc;
                z = fb / fc;
                x = sv * (2.0 * xm * y * (y - z) - (b - a) * (z - 1.0));
                y = (y - 1.0) * (z - 1.0) * (sv - 1.0);
            }
            if (x > 0.0) y = -y;
            x = fabs(x);
            const double m1 = 3.0 * xm * y - fabs(E_crit * y), m2 = fabs(e * y);
            if (2.0 * x < (m1 < m2 ? m1 : m2)) { e = d; d = x / y; }
            else { d = xm; e = d; }
        } else { d = xm; e = d; }
        a = b;
        fa = fb;
        if (fabs(d) > E_crit) b = b + d;
        else b = b + (xm >= 0.0 ? E_crit : -E_crit);
        fb = H(b);
    }
    if (threadIdx.x == 0) {
        if (!ok) atomicOr(status, ST_LINE_NOBRACKET);
        const double err = acc[A_PMAX] * fabs(alpha);          // ctip.f90:187
        line[L_ALPHA] = alpha;
        line[L_ERROR] = err;
        line[L_DONE] = err > ecrit ? 0.0 : 1.0;
        line[L_NEVAL] += (double)(2 + (ok ? n - 1 : 100));
        line[L_GSUM_OLD] = acc[A_GSUM];
        acc[A_GSUM] = 0.0;
        acc[A_PSUM] = 0.0;
        acc[A_PMAX] = 0.0;
        acc[A_GP] = 0.0;
        acc[A_PAP] = 0.0;
    }
}

// The same Brent iteration with each h(b) spread over the whole GPU: every
// CTA runs the identical control flow, sums its slice of the active set, and
// a grid barrier exchanges the per-CTA partial sums, which every CTA then
// adds in CTA order -- so all CTAs see the same h(b), take the same branches
// and agree on the returned b.  Launched cooperatively, so all CTAs are
// resident; each barrier wait still gives up after a bounded number of polls
// (ST_SYNC), after which the kernel skips its remaining waits and ends.
constexpr int BR_THREADS = 256;
constexpr long long kBarrierPolls = 1LL << 22;

// Grid barrier on (count, gen): returns false when the wait gave up.
__device__ __forceinline__ bool grid_barrier(unsigned* count, unsigned* gen, unsigned nb, int& ok_sh) {
    __syncthreads();
    if (threadIdx.x == 0) {
        int ok = 1;
        const unsigned g = atomicAdd(gen, 0u);
        __threadfence();
        if (atomicAdd(count, 1u) == nb - 1u) {
            atomicExch(count, 0u);
            __threadfence();
            atomicAdd(gen, 1u);
        } else {
            long long it = 0;
            while (atomicAdd(gen, 0u) == g) {
                if (++it > kBarrierPolls) {
                    ok = 0;
                    break;
                }
                __nanosleep(64);
            }
        }
        __threadfence();
        ok_sh = ok;
    }
    __syncthreads();
    return ok_sh != 0;
}

__global__ void __launch_bounds__(BR_THREADS)
    ctip_brent_grid_kernel(const int* __restrict__ ts, const double* __restrict__ q, const double* __restrict__ pv,
                           const int* __restrict__ act, const int* __restrict__ nact, CtipSpecies S,
                           double* __restrict__ line, double* __restrict__ acc, double ecrit, int* __restrict__ status,
                           double* __restrict__ part, unsigned* __restrict__ bar) {
    __shared__ double red[BR_THREADS / 32];
    __shared__ double tot;
    __shared__ int ok_sh;
    const double gp = acc[A_GP], pap = acc[A_PAP];
    const int na = *nact;
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const unsigned nb = gridDim.x;
    bool synced = true;
    int ev = 0;
    auto H = [&](double b) -> double {
        double s = 0.0;
        for (int k = blockIdx.x * BR_THREADS + threadIdx.x; k < na; k += nb * BR_THREADS) {
            const int i = act[k];
            const int sp = min(ts[i], 4);
            const double qi = q[i], p = pv[i];
            s += p * (pen_d(qi + b * p, S.qmin[sp], S.qmax[sp]) - pen_d(qi, S.qmin[sp], S.qmax[sp]));
        }
        s = warp_sum(s);
        if (lane == 0) red[w] = s;
        __syncthreads();
        double* slot = part + (ev & 1) * nb;
        if (threadIdx.x == 0) {
            double t = 0.0;
            for (int j = 0; j < BR_THREADS / 32; j++) t += red[j];
            slot[blockIdx.x] = t;
        }
        ev++;
        if (synced) synced = grid_barrier(bar, bar + 1, nb, ok_sh);
        if (threadIdx.x == 0) {
            double t = 0.0;
            for (unsigned j = 0; j < nb; j++) t += *(volatile double*)(slot + j);   // CTA order: same in every CTA
            tot = t;
        }
        __syncthreads();
        const double h = -gp + b * pap + tot;   // = -sum g(q + b p) p
        __syncthreads();
        return synced ? h : NAN;
    };
    const double E_crit = 1.0e-8, E_end = 1.0e-11;
    double a = -1.0, b = 1.0, c, d = 0.0, e = 0.0, fa, fb, fc, xm, sv, x, y, z;
    fa = H(a);
    fb = H(b);
    c = b;
    fc = fb;
    double alpha = b;
    int n, ok = 0;
    for (n = 1; n <= 100; n++) {
        if ((fb > 0.0 && fc > 0.0) || (fb < 0.0 && fc < 0.0)) { c = a; fc = fa; d = b - a; e = d; }
        if (fabs(fc) < fabs(fb)) { a = b; b = c; c = a; fa = fb; fb = fc; fc = fa; }
        xm = 0.5 * (c - b);
        if (fabs(xm) < E_crit || fabs(fb) < E_end) { alpha = b; ok = 1; break; }
        if (fabs(e) >= E_crit && fabs(fa) > fabs(fb)) {
            sv = fb / fa;
            if (a == c) { x = 2.0 * xm * sv; y = 1.0 - sv; }
            else {
                y = fa / fc;
                z = fb / fc;
                x = sv * (2.0 * xm * y * (y - z) - (b - a) * (z - 1.0));
                y = (y - 1.0) * (z - 1.0) * (sv - 1.0);
            }
            if (x > 0.0) y = -y;
            x = fabs(x);
            const double m1 = 3.0 * xm * y - fabs(E_crit * y), m2 = fabs(e * y);
            if (2.0 * x < (m1 < m2 ? m1 : m2)) { e = d; d = x / y; }
            else { d = xm; e = d; }
        } else { d = xm; e = d; }
        a = b;
        fa = fb;
        if (fabs(d) > E_crit) b = b + d;
        else b = b + (xm >= 0.0 ? E_crit : -E_crit);
        fb = H(b);
        if (!synced) break;
    }
    if (!synced) {
        if (threadIdx.x == 0) atomicOr(status, ST_SYNC);
        return;
    }
    // every CTA has read gp, pap and the partials of its last evaluation
    // before any CTA left the last barrier; CTA 0 writes the results
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        if (!ok) atomicOr(status, ST_LINE_NOBRACKET);
        const double err = acc[A_PMAX] * fabs(alpha);          // ctip.f90:187
        line[L_ALPHA] = alpha;
        line[L_ERROR] = err;
        line[L_DONE] = err > ecrit ? 0.0 : 1.0;
        line[L_NEVAL] += (double)(2 + (ok ? n - 1 : 100));
        line[L_GSUM_OLD] = acc[A_GSUM];
        acc[A_GSUM] = 0.0;
        acc[A_PSUM] = 0.0;
        acc[A_PMAX] = 0.0;
        acc[A_GP] = 0.0;
        acc[A_PAP] = 0.0;
    }
}

// q += alpha p; g -= alpha Ap + dpen; sum g   (ctip.f90:185 and the next dUdq)
__global__ void __launch_bounds__(CT_THREADS)
    ctip_update_kernel(int n, const int* __restrict__ ts, double* __restrict__ q, double* __restrict__ g,
                       const double* __restrict__ pv, const double* __restrict__ Ap, CtipSpecies S,
                       const double* __restrict__ line, double* __restrict__ acc) {
    __shared__ double red[CT_THREADS / 32];
    const double alpha = line[L_ALPHA];
    double gs = 0.0;
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) {
        const int s = min(ts[i], 4);
        const double q0 = q[i];
        const double q1 = q0 + alpha * pv[i];
        const double gn = g[i] - alpha * Ap[i] - (pen_d(q1, S.qmin[s], S.qmax[s]) - pen_d(q0, S.qmin[s], S.qmax[s]));
        q[i] = q1;
        g[i] = gn;
        gs = gn;
    }
    block_add<CT_THREADS>(gs, acc, A_GSUM, red);
}

// write charges back (original order and the sorted copy); Eself pieces (ctip.f90:194-209)
__global__ void __launch_bounds__(CT_THREADS)
    ctip_final_kernel(int n, const int* __restrict__ ts, const int* __restrict__ sorted, const double* __restrict__ qs,
                      double* __restrict__ q, double4* __restrict__ xq, float4* __restrict__ frec,
                      double4* __restrict__ xo, CtipSpecies S, double* __restrict__ acc) {
    __shared__ double red[CT_THREADS / 32];
    double q2 = 0.0, es = 0.0, qsum = 0.0;
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) {
        const int s = min(ts[i], 4);
        const double qi = qs[i];
        q[sorted[i]] = qi;
        xq[i].w = qi;
        frec[i].w = (float)qi;   // skin-mode force records (unused otherwise)
        xo[i].w = qi;
        q2 = -(qi * qi);
        qsum = qi;
        es = S.chi[s] * qi + 0.5 * S.Jp[s] * (qi * qi);
        double dq = qi - S.qmin[s];
        if (dq < 0.0) es += SX_WPEN * (dq * dq);
        dq = qi - S.qmax[s];
        if (dq > 0.0) es += SX_WPEN * (dq * dq);
    }
    block_add<CT_THREADS>(q2, acc, A_Q2SUM, red);
    block_add<CT_THREADS>(es, acc, A_ESUM, red);
    block_add<CT_THREADS>(qsum, acc, A_QSUM, red);
}

__global__ void copy_q_sorted_kernel(int n, const double4* __restrict__ xq, double* __restrict__ qs) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) qs[i] = xq[i].w;
}

// ---------------------------------------------------------------------------
int ctip_alloc(simox_ctx* c) {
    const size_t N = (size_t)std::max(c->cap, 1);
    bool ok = cudaMalloc(&c->c_const, N * sizeof(double)) == cudaSuccess &&
              cudaMalloc(&c->g, N * sizeof(double)) == cudaSuccess &&
              cudaMalloc(&c->pv, N * sizeof(double)) == cudaSuccess &&
              cudaMalloc(&c->Ap, N * sizeof(double)) == cudaSuccess &&
              cudaMalloc(&c->qs, N * sizeof(double)) == cudaSuccess &&
              cudaMalloc(&c->jp, N * sizeof(double)) == cudaSuccess &&       // short-range product scratch
              cudaMalloc(&c->act, (N + 1) * sizeof(int)) == cudaSuccess;
    return ok ? SIMOX_OK : SIMOX_E_NOMEM;
}

CtipSpecies ctip_species(const simox_ctx* c) {
    CtipSpecies S;
    const double kc_const = SX_KC * 2.0 * c->a / SX_SQRTPI;   // ctip.f90:31
    for (int s = 0; s < 5; s++) {
        const simox_potn& p = c->pot.param[s];
        S.chi[s] = p.chi;
        S.Jp[s] = p.J - kc_const;                               // ctip.f90:37
        S.qmin[s] = p.qmin;
        S.qmax[s] = p.qmax;
        S.Z[s] = p.Z;
    }
    return S;
}

template <typename R>
static void launch_ctip_pair(simox_ctx* c, const PairTab<R>* tab, const double* vin, double* out, double* cconst,
                             const CtipSpecies& S) {
    CtipParams P;
    P.box = make_double3(c->box[0], c->box[1], c->box[2]);
    P.ibox = make_double3(c->inv_box[0], c->inv_box[1], c->inv_box[2]);
    P.a = c->a;
    P.kc = SX_KC;
    P.cap = c->nnb_cap;
    P.n = c->n;
    int wpb = CT_THREADS / 32;
    int g = std::min((c->n + wpb - 1) / wpb, num_sms(c) * 8);
    if (g < 1) g = 1;
    if (cconst)
        ctip_pair_kernel<R, true><<<g, CT_THREADS, 0, c->stream>>>(P, tab, c->xq_s, c->t_s, reinterpret_cast<const int2*>(c->nn), c->nbr, vin, out,
                                                                   cconst, S);
    else
        ctip_pair_kernel<R, false><<<g, CT_THREADS, 0, c->stream>>>(P, tab, c->xq_s, c->t_s, reinterpret_cast<const int2*>(c->nn), c->nbr, vin, out,
                                                                    nullptr, S);
}

void ctip_pair(simox_ctx* c, const double* vin, double* out, double* cconst, const CtipSpecies& S) {
    Launch L(c, cconst ? "ctip_setup_pairs" : "ctip_matvec_pairs");
    if (c->precision == SIMOX_MIXED && half_path(c)) {   // a launch error surfaces at the next check
        ctip_pair_half(c, vin, out, cconst, S);
        return;
    }
    if (c->precision == SIMOX_MIXED) launch_ctip_pair<float>(c, c->tab_f, vin, out, cconst, S);
    else launch_ctip_pair<double>(c, c->tab_d, vin, out, cconst, S);
}

// The line search on the whole GPU (cooperative launch, one CTA per SM); false
// when that launch is not available here (the caller then runs the one-CTA
// kernel).  Scratch: the per-CTA partial sums in the short-range work vector
// (free during the line search) and the barrier words in the line slots.
static bool brent_grid(simox_ctx* c, const CtipSpecies& S, double tol, int* nact) {
    if (!c->coop_brent) return false;
    const int nbk = num_sms(c);
    if ((size_t)2 * nbk > (size_t)c->cap) return false;
    unsigned* bar = reinterpret_cast<unsigned*>(c->line + 62);
    cudaMemsetAsync(bar, 0, 2 * sizeof(unsigned), c->stream);
    cudaLaunchConfig_t cfg{};
    cfg.gridDim = dim3(nbk);
    cfg.blockDim = dim3(BR_THREADS);
    cfg.stream = c->stream;
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeCooperative;
    at[0].val.cooperative = 1;
    cfg.attrs = at;
    cfg.numAttrs = 1;
    const cudaError_t e = cudaLaunchKernelEx(&cfg, ctip_brent_grid_kernel, (const int*)c->t_s, (const double*)c->qs,
                                             (const double*)c->pv, (const int*)c->act, (const int*)nact, S, c->line,
                                             c->acc, tol, c->status, c->jp, bar);
    if (e != cudaSuccess) {
        cudaGetLastError();
        c->coop_brent = false;
        return false;
    }
    return true;
}

// One nonlinear-CG iteration (ctip.f90:169-190): direction with the
// reference's beta, mean projection, A p (PME potential + short-range pairs),
// the Brent line search and the update.  Every launch goes to c->stream, so
// the iteration can be captured into a graph body.
static int ctip_iteration(simox_ctx* c, const CtipSpecies& S, double c_pme, double tol, int* nact, int nb) {
    const int n = c->n;
    cudaStream_t s = c->stream;
    cudaMemsetAsync(nact, 0, sizeof(int), s);
    {
        Launch L(c, "ctip_direction");
        ctip_dir_kernel<<<nb, CT_THREADS, 0, s>>>(n, c->g, c->pv, c->line, c->acc);
    }
    {
        Launch L(c, "ctip_project");
        ctip_proj_kernel<<<nb, CT_THREADS, 0, s>>>(n, c->pv, c->acc);
    }
    if (c->precision == SIMOX_MIXED && half_path(c)) {
        // A p as one fused product: the half-list pair sums run on the side
        // stream while the main stream spreads p and transforms the grid;
        // one kernel then gathers the potential and adds the pair sums, J' p,
        // the dots and the active set
        cudaMemsetAsync(c->fx_acc, 0, sizeof(unsigned long long) * (size_t)n, s);
        cudaStream_t ps = c->profiling ? s : c->side;   // profiled launches stay on one stream
        if (ps != s) {
            cudaEventRecord(c->ev_fork, s);
            cudaStreamWaitEvent(ps, c->ev_fork, 0);
        }
        if (int st = ctip_half_launch(c, c->pv, ps)) return st;
        if (ps != s) cudaEventRecord(c->ev_join, ps);
        if (int st = pme_potential_grid(c, c->pv)) return st;
        if (ps != s) cudaStreamWaitEvent(s, c->ev_join, 0);
        CtipFinish F{c->t_s, c->qs, c->g, c->pv, c->fx_acc, ctip_half_unit(), c->Ap, c->act, nact, c->acc, S};
        if (int st = pme_potential_finish(c, c_pme, F)) return st;
    } else {
        if (int st = pme_potential(c, c->pv, c->Ap, c_pme)) return st;
        ctip_pair(c, c->pv, c->jp, nullptr, S);
        Launch L(c, "ctip_matvec_finish");
        ctip_matvec_finish_kernel<<<nb, CT_THREADS, 0, s>>>(n, c->t_s, c->qs, c->g, c->pv, c->jp, c->Ap, S, c->act,
                                                           nact, c->acc);
    }
    {
        Launch L(c, "ctip_brent");
        if (!brent_grid(c, S, tol, nact))
            ctip_brent_kernel<<<1, 1024, 0, s>>>(c->t_s, c->qs, c->pv, c->act, nact, S, c->line, c->acc, tol,
                                                 c->status);
    }
    {
        Launch L(c, "ctip_update");
        ctip_update_kernel<<<nb, CT_THREADS, 0, s>>>(n, c->t_s, c->qs, c->g, c->pv, c->Ap, S, c->line, c->acc);
    }
    return check_launch(c);
}

// Device-side loop: the iteration is the body of a CUDA graph WHILE node whose
// condition this kernel sets after every iteration.  One graph launch runs at
// most kCgChunk iterations, so every launch ends after a bounded time and the
// host checks the status between launches.
constexpr int kCgChunk = 256;

__global__ void ctip_loop_cond_kernel(cudaGraphConditionalHandle h, double* __restrict__ line,
                                      const int* __restrict__ status, int max_cg, int chunk) {
    const double k = line[L_ITERS] + 1.0;
    const double kc = line[L_CHUNK] + 1.0;
    line[L_ITERS] = k;
    line[L_CHUNK] = kc;
    const bool stop = line[L_DONE] != 0.0 || *status != 0 || !isfinite(line[L_ERROR]) ||
                      (max_cg > 0 && k >= (double)max_cg) || kc >= (double)chunk;
    cudaGraphSetConditional(h, stop ? 0u : 1u);
}

// Runs the CG loop as graph launches.  *used = false (nothing run) when the
// graph cannot be built here; the caller then runs the host-driven loop.
static int ctip_device_loop(simox_ctx* c, const CtipSpecies& S, double c_pme, double tol, int* nact, int nb,
                            int max_cg, int* k_out, double hbuf[4], bool* used) {
    *used = false;
    cudaStream_t s = c->stream;
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
            st = ctip_iteration(c, S, c_pme, tol, nact, nb);
            ctip_loop_cond_kernel<<<1, 1, 0, s>>>(h, c->line, c->status, max_cg, kCgChunk);
            cudaGraph_t cap = nullptr;
            ok = cudaStreamEndCapture(s, &cap) == cudaSuccess && st == SIMOX_OK;
            per_iter = c->launches - l0 + 1;
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
    double lb[6] = {0.0, 1.0, 0.0, 0.0, 0.0, 0.0};
    int k = 0;
    while (true) {
        cudaMemsetAsync(c->line + L_CHUNK, 0, sizeof(double), s);
        if ((st = cuda_status(cudaGraphLaunch(exec, s)))) break;
        cudaMemcpyAsync(lb, c->line + L_ALPHA, sizeof(double) * 6, cudaMemcpyDeviceToHost, s);
        cudaMemcpyAsync(c->h_status, c->status, sizeof(int), cudaMemcpyDeviceToHost, s);
        if ((st = cuda_status(cudaStreamSynchronize(s)))) break;
        const int k_now = (int)lb[4];
        c->launches += per_iter * (long long)(k_now - k);
        k = k_now;
        if (*c->h_status || lb[2] != 0.0 || !std::isfinite(lb[1]) || (max_cg > 0 && k >= max_cg)) break;
    }
    for (int i = 0; i < 4; i++) hbuf[i] = lb[i];
    *k_out = k;
    cudaGraphExecDestroy(exec);
    cudaGraphDestroy(outer);
    return st;
}

int ctip_solve(simox_ctx* c, int max_cg, simox_ctip_report* rep, double tol) {
    if (!c->psi_valid) return SIMOX_E_STATE;
    int st = ensure_list(c);
    if (st) return st;
    if ((st = read_status(c))) return st;
    const int n = c->n;
    if (n == 0) return SIMOX_OK;
    const CtipSpecies S = ctip_species(c);
    const double V = c->box[0] * c->box[1] * c->box[2];
    const double c_pme = SX_KC * (double)c->fft[0] * (double)c->fft[1] * (double)c->fft[2] / V / SX_PI;  // ctip.f90:59
    const int nb = (n + CT_THREADS - 1) / CT_THREADS;
    int* nact = c->act + c->cap;
    cudaStream_t s = c->stream;
    cudaMemsetAsync(c->acc + A_GSUM, 0, sizeof(double) * (A_LINE0 - A_GSUM), s);
    cudaMemsetAsync(c->line, 0, sizeof(double) * L_END, s);
    {
        Launch L(c, "ctip_copy_q");
        copy_q_sorted_kernel<<<nb, CT_THREADS, 0, s>>>(n, c->xq_s, c->qs);
    }
    // gsum_old = 1 (ctip.f90:168)
    const double one = 1.0;
    cudaMemcpyAsync(c->line + L_GSUM_OLD, &one, sizeof(double), cudaMemcpyHostToDevice, s);
    // g0 = -(chi + sum Z asym + J'q + phi(q) + pen'(q) + sum sym q)
    ctip_pair(c, c->qs, c->jp, c->c_const, S);
    if ((st = pme_potential(c, c->qs, c->g, c_pme))) return st;
    {
        Launch L(c, "ctip_init");
        ctip_init_g_kernel<<<nb, CT_THREADS, 0, s>>>(n, c->t_s, c->qs, c->c_const, c->jp, c->g, c->pv, S, c->acc);
    }
    int k = 0;
    double err = 1.0;
    double hbuf[4] = {0.0, 1.0, 0.0, 0.0};
    bool device_loop = false;
    if (!c->profiling && (st = ctip_device_loop(c, S, c_pme, tol, nact, nb, max_cg, &k, hbuf, &device_loop))) return st;
    if (device_loop) {
        err = hbuf[1];
        if (*c->h_status) st = read_status(c);                            // Brent limit (ctip.f90:302)
        else if (!std::isfinite(err)) st = SIMOX_E_BRENT;
        else if (hbuf[2] == 0.0 && max_cg > 0 && k >= max_cg) st = SIMOX_E_CG_LIMIT;
    }
    while (!device_loop) {
        if (max_cg > 0 && k >= max_cg) { st = SIMOX_E_CG_LIMIT; break; }
        if ((st = ctip_iteration(c, S, c_pme, tol, nact, nb))) return st;
        k++;
        cudaMemcpyAsync(hbuf, c->line + L_ALPHA, sizeof(double) * 4, cudaMemcpyDeviceToHost, s);
        cudaMemcpyAsync(c->h_status, c->status, sizeof(int), cudaMemcpyDeviceToHost, s);
        if ((st = cuda_status(cudaStreamSynchronize(s)))) return st;
        err = hbuf[1];
        if (*c->h_status) { st = read_status(c); break; }   // Brent limit (ctip.f90:302)
        if (hbuf[2] != 0.0) break;
        if (!std::isfinite(err)) { st = SIMOX_E_BRENT; break; }
    }
    if (st && st != SIMOX_E_CG_LIMIT) return st;
    cudaMemsetAsync(c->acc + A_Q2SUM, 0, 2 * sizeof(double), s);
    cudaMemsetAsync(c->acc + A_QSUM, 0, sizeof(double), s);
    {
        Launch L(c, "ctip_final");
        ctip_final_kernel<<<nb, CT_THREADS, 0, s>>>(n, c->t_s, c->pair_order, c->qs, c->q, c->xq_s, c->frec_s, c->xo_s, S,
                                                              c->acc);
    }
    cudaMemcpyAsync(c->h_acc, c->acc, sizeof(double) * A_COUNT, cudaMemcpyDeviceToHost, s);
    int s2 = cuda_status(cudaStreamSynchronize(s));
    if (s2) return s2;
    c->eam_valid = false;   // charges changed: forces must be recomputed
    // ctip.f90:209  Eself = Eself*kc*a/SQRTPI + Esum
    c->eself = c->h_acc[A_Q2SUM] * SX_KC * c->a / SX_SQRTPI + c->h_acc[A_ESUM];
    if (rep) {
        rep->n_cg = k;
        rep->n_line = (int)hbuf[3];
        rep->error = err;
        rep->q_sum = c->h_acc[A_QSUM];
    }
    return st;
}

}  // namespace sx
