// integrate.cu -- velocity-Verlet kernels of vverlet.f90.
//
// Each kernel reproduces the reference's FP64 operation order with explicit
// round-to-nearest intrinsics (no FMA contraction), so given the same forces
// the positions and velocities are bit-identical to the Fortran statements:
//   VV_NVE1         vverlet.f90:74-96    v += 0.5 dt f/m; x += dt v; x -= L DNINT(x/L)
//   VV_NVE1_REFLECT vverlet.f90:100-129  same, z reflected at +L/2 instead of wrapped
//   VV_NVE2         vverlet.f90:132-157  v += 0.5 dt f/m; mv2 = sum m v^2
//   VV_NVT2_BEREND  vverlet.f90:160-208  half kick, per-species T, v *= lambda_s
//   VV_NVT1_STOCH   vverlet.f90:237-260  damped half kick, drift, wrap
//   VV_NVT2_STOCH   vverlet.f90:263-296  random force, damped half kick
//   VINIT           vverlet.f90:2-71     seeded velocities at T_given
// The second half kick optionally first removes the mean PME force
// (force.f90:457-460), f = f - Fsum/N, and stores the final force.
#include "simox_internal.cuh"

#include <cmath>

namespace sx {

struct Masses { double xm[5]; };

__device__ __forceinline__ double half_kick(double v, double f, double dt, double xm) {
    return __dadd_rn(v, __ddiv_rn(__dmul_rn(__dmul_rn(0.5, dt), f), xm));
}

__device__ __forceinline__ void vv1_body(Blk B, int n, const int* __restrict__ id, double* __restrict__ x,
                                         double* __restrict__ v, const double* __restrict__ f, double dt, double3 box,
                                         const Masses& M, int reflect) {
    const int i = B.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const double xm = M.xm[id[i] - 1];
    const double L[3] = {box.x, box.y, box.z};
    double xx[3];
#pragma unroll
    for (int d = 0; d < 3; d++) {
        const double vv = half_kick(v[3 * i + d], f[3 * i + d], dt, xm);
        v[3 * i + d] = vv;
        xx[d] = __dadd_rn(x[3 * i + d], __dmul_rn(dt, vv));
    }
    const int nwrap = reflect ? 2 : 3;
#pragma unroll
    for (int d = 0; d < 3; d++) {
        if (d < nwrap) x[3 * i + d] = __dsub_rn(xx[d], __dmul_rn(L[d], round(__ddiv_rn(xx[d], L[d]))));
    }
    if (reflect) {
        double z = xx[2];
        if (z > box.z / 2.0) {
            z = __dsub_rn(box.z, z);
            v[3 * i + 2] = -fabs(v[3 * i + 2]);
        }
        x[3 * i + 2] = z;
    }
}
__global__ void __launch_bounds__(256) vv1_kernel(int n, const int* __restrict__ id, double* __restrict__ x,
                                                  double* __restrict__ v, const double* __restrict__ f, double dt,
                                                  double3 box, const __grid_constant__ Masses M, int reflect) {
    vv1_body(own_blk(), n, id, x, v, f, dt, box, M, reflect);
}

// second half kick (+ optional mean-force removal); mv2 and per-species sums
template <bool BEREND>
__device__ __forceinline__ void vv2_body(Blk B, int n, const int* __restrict__ id, double* __restrict__ v,
                                         double* __restrict__ f, const double* __restrict__ f_add, double dt,
                                         const Masses& M, double* __restrict__ acc, int subtract_mean) {
    __shared__ double red[256 / 32];
    double mv2 = 0.0;
    double ms[5] = {0, 0, 0, 0, 0};
    double ns[5] = {0, 0, 0, 0, 0};
    const int i = B.x * blockDim.x + threadIdx.x;
    if (i < n) {
        const int s = id[i] - 1;
        const double xm = M.xm[s];
        double t = 0.0;
#pragma unroll
        for (int d = 0; d < 3; d++) {
            double ff = f[3 * i + d];
            if (f_add) ff = __dadd_rn(ff, f_add[3 * i + d]);   // ff + ff_rec - Fsum (force.f90:459)
            if (subtract_mean) ff = __dsub_rn(ff, __ddiv_rn(acc[A_FSUM0 + d], (double)n));
            if (f_add || subtract_mean) f[3 * i + d] = ff;
            const double vv = half_kick(v[3 * i + d], ff, dt, xm);
            v[3 * i + d] = vv;
            if (BEREND) t = __dadd_rn(t, __dmul_rn(xm, __dmul_rn(vv, vv)));
            else t = __dadd_rn(t, __dmul_rn(vv, vv));
        }
        if (BEREND) {
#pragma unroll
            for (int k = 0; k < 5; k++)
                if (k == s) { ms[k] = t; ns[k] = 1.0; }
        } else {
            mv2 = __dmul_rn(xm, t);
        }
    }
    if (BEREND) {
#pragma unroll
        for (int k = 0; k < 5; k++) {
            block_add<256>(ms[k], acc, A_MV2S0 + k, red);
            block_add<256>(ns[k], acc, A_NS0 + k, red);
        }
    } else {
        block_add<256>(mv2, acc, A_MV2, red);
    }
}
template <bool BEREND>
__global__ void __launch_bounds__(256)
    vv2_kernel(int n, const int* __restrict__ id, double* __restrict__ v, double* __restrict__ f,
               const double* __restrict__ f_add, double dt, const __grid_constant__ Masses M,
               double* __restrict__ acc, int subtract_mean) {
    vv2_body<BEREND>(own_blk(), n, id, v, f, f_add, dt, M, acc, subtract_mean);
}

// Berendsen rescale (vverlet.f90:188-205)
__device__ __forceinline__ void berend_scale_body(Blk B, int n, const int* __restrict__ id, double* __restrict__ v,
                                                  const Masses& M, double T_given, double* __restrict__ acc) {
    __shared__ double red[256 / 32];
    __shared__ double lam[5];
    if (threadIdx.x < 5) {
        const int k = threadIdx.x;
        double l = 0.0;
        const double np = acc[A_NS0 + k];
        if (np > 0.0) {
            const double T0 = acc[A_MV2S0 + k] / (3.0 * np);
            l = sqrt(1.0 + 0.025 * (T_given / T0 - 1.0));
        }
        lam[k] = l;
    }
    __syncthreads();
    double mv2 = 0.0;
    const int i = B.x * blockDim.x + threadIdx.x;
    if (i < n) {
        const int s = id[i] - 1;
        const double xm = M.xm[s];
        double t = 0.0;
#pragma unroll
        for (int d = 0; d < 3; d++) {
            const double vv = __dmul_rn(v[3 * i + d], lam[s]);
            v[3 * i + d] = vv;
            t = __dadd_rn(t, __dmul_rn(xm, __dmul_rn(vv, vv)));
        }
        mv2 = t;
    }
    block_add<256>(mv2, acc, A_MV2, red);
}
__global__ void __launch_bounds__(256)
    berend_scale_kernel(int n, const int* __restrict__ id, double* __restrict__ v, const __grid_constant__ Masses M,
                        double T_given, double* __restrict__ acc) {
    berend_scale_body(own_blk(), n, id, v, M, T_given, acc);
}

// ---------------------------------------------------------------------------
// VINIT and the stochastic thermostat.  The reference draws from Fortran's
// RANDOM_NUMBER (main.f90:28 RANDOM_SEED), which nothing else can reproduce;
// here every draw is a pure function of (seed, stream, counter): the
// SplitMix64 output mix (Steele, Lea & Flood, OOPSLA 2014) applied twice,
// 53 bits scaled into [0, 1).  Streams: VINIT (1 << 62 | atom), counter =
// component; thermostat (step << 32 | atom), counters 2 (256 d + k) and
// 2 (256 d + k) + 1 for attempt k of component d.  Atom = original index.
__device__ __forceinline__ unsigned long long mix64(unsigned long long z) {
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
    return z ^ (z >> 31);
}
__device__ __forceinline__ double rng_uniform(unsigned long long seed, unsigned long long a, unsigned long long b) {
    const unsigned long long g = 0x9E3779B97F4A7C15ULL;
    const unsigned long long z = mix64(mix64(seed + g * (a + 1)) + g * (b + 1));
    return (double)(z >> 11) * (1.0 / 9007199254740992.0);
}

// fluct (util.f90:84-101) with x = 1: Marsaglia's polar method, v1 kept.  At
// most 100 attempts (each rejected with probability 1 - pi/4); after that 0
// and *bad.
__device__ double fluct_draw(unsigned long long seed, unsigned long long step, int i, int d, int& bad) {
    const unsigned long long a = (step << 32) | (unsigned long long)(unsigned)i;
    for (int k = 0; k < 100; k++) {
        const unsigned long long b = 2ULL * (unsigned long long)(256 * d + k);
        const double v1 = __dsub_rn(__dmul_rn(2.0, rng_uniform(seed, a, b)), 1.0);
        const double v2 = __dsub_rn(__dmul_rn(2.0, rng_uniform(seed, a, b + 1)), 1.0);
        const double r = __dadd_rn(__dmul_rn(v1, v1), __dmul_rn(v2, v2));
        if (r < 1.0 && r > 0.0) return __dmul_rn(v1, sqrt(__ddiv_rn(__dmul_rn(-2.0, log(r)), r)));
    }
    bad = 1;
    return 0.0;
}

// VINIT (vverlet.f90:19-27): v = U[0,1) - 0.5 per component, sums per axis
__global__ void __launch_bounds__(256)
    vinit_draw_kernel(int n, unsigned long long seed, double* __restrict__ v, double* __restrict__ acc) {
    __shared__ double red[256 / 32];
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    double s[3] = {0.0, 0.0, 0.0};
    if (i < n) {
#pragma unroll
        for (int d = 0; d < 3; d++) {
            s[d] = __dsub_rn(rng_uniform(seed, (1ULL << 62) | (unsigned long long)(unsigned)i, (unsigned long long)d),
                             0.5);
            v[3 * i + d] = s[d];
        }
    }
#pragma unroll
    for (int d = 0; d < 3; d++) block_add<256>(s[d], acc, A_LINE0 + d, red);
}

// VINIT (vverlet.f90:29-38): mean removed; per-species m v^2 and counts
__global__ void __launch_bounds__(256)
    vinit_center_kernel(int n, const int* __restrict__ id, double* __restrict__ v, Masses M,
                        double* __restrict__ acc) {
    __shared__ double red[256 / 32];
    double ms[5] = {0, 0, 0, 0, 0}, ns[5] = {0, 0, 0, 0, 0};
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) {
        const int s = id[i] - 1;
        double w[3];
#pragma unroll
        for (int d = 0; d < 3; d++) {
            w[d] = __dsub_rn(v[3 * i + d], __ddiv_rn(acc[A_LINE0 + d], (double)n));
            v[3 * i + d] = w[d];
        }
        const double t =
            __dmul_rn(M.xm[s], __dadd_rn(__dadd_rn(__dmul_rn(w[0], w[0]), __dmul_rn(w[1], w[1])), __dmul_rn(w[2], w[2])));
#pragma unroll
        for (int k = 0; k < 5; k++)
            if (k == s) { ms[k] = t; ns[k] = 1.0; }
    }
#pragma unroll
    for (int k = 0; k < 5; k++) {
        block_add<256>(ms[k], acc, A_MV2S0 + k, red);
        block_add<256>(ns[k], acc, A_NS0 + k, red);
    }
}

// VINIT (vverlet.f90:40-55, 64-69): v *= sqrt(T_given / T0_s); the as-written
// mv2 multiplies every atom's v^2 by the mass the earlier loop left in xm,
// the last atom's.
__global__ void __launch_bounds__(256)
    vinit_scale_kernel(int n, const int* __restrict__ id, double* __restrict__ v, Masses M, double T_given,
                       double* __restrict__ acc) {
    __shared__ double red[256 / 32];
    __shared__ double lam[5];
    if (threadIdx.x < 5) {
        const int k = threadIdx.x;
        const double np = acc[A_NS0 + k];
        lam[k] = np > 0.0 ? sqrt(__ddiv_rn(T_given, __ddiv_rn(acc[A_MV2S0 + k], 3.0 * np))) : 0.0;
    }
    __syncthreads();
    double mv2 = 0.0;
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) {
        const double xm_last = M.xm[id[n - 1] - 1];
        const int s = id[i] - 1;
        double w[3];
#pragma unroll
        for (int d = 0; d < 3; d++) {
            w[d] = __dmul_rn(v[3 * i + d], lam[s]);
            v[3 * i + d] = w[d];
        }
        mv2 = __dmul_rn(xm_last,
                        __dadd_rn(__dadd_rn(__dmul_rn(w[0], w[0]), __dmul_rn(w[1], w[1])), __dmul_rn(w[2], w[2])));
    }
    block_add<256>(mv2, acc, A_MV2, red);
}

// VV_NVT1_STOCH (vverlet.f90:237-260): v = v (1 - alpha dt / 2m) + dt f / 2m,
// x += dt v, wrapped
__global__ void vv1_stoch_kernel(int n, const int* __restrict__ id, double* __restrict__ x, double* __restrict__ v,
                                 const double* __restrict__ f, double dt, double alpha, double3 box, Masses M) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const double xm = M.xm[id[i] - 1];
    const double damp = __dsub_rn(1.0, __ddiv_rn(__dmul_rn(__dmul_rn(0.5, alpha), dt), xm));
    const double L[3] = {box.x, box.y, box.z};
#pragma unroll
    for (int d = 0; d < 3; d++) {
        const double vv = __dadd_rn(__dmul_rn(v[3 * i + d], damp),
                                    __ddiv_rn(__dmul_rn(__dmul_rn(0.5, dt), f[3 * i + d]), xm));
        v[3 * i + d] = vv;
        const double xx = __dadd_rn(x[3 * i + d], __dmul_rn(dt, vv));
        x[3 * i + d] = __dsub_rn(xx, __dmul_rn(L[d], round(__ddiv_rn(xx, L[d]))));
    }
}

// VV_NVT2_STOCH (vverlet.f90:263-296): f += eta beta, v = (v + dt f / 2m) /
// (1 + alpha dt / 2m), mv2 = sum m v^2.  f first gains f_add and loses the
// mean force as in vv2_kernel.
__global__ void __launch_bounds__(256)
    vv2_stoch_kernel(int n, const int* __restrict__ id, double* __restrict__ v, double* __restrict__ f,
                     const double* __restrict__ f_add, double dt, double alpha, double beta, unsigned long long seed,
                     unsigned long long step, Masses M, double* __restrict__ acc, int subtract_mean,
                     int* __restrict__ status) {
    __shared__ double red[256 / 32];
    double mv2 = 0.0;
    int bad = 0;
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) {
        const double xm = M.xm[id[i] - 1];
        const double den = __dadd_rn(1.0, __ddiv_rn(__dmul_rn(__dmul_rn(0.5, alpha), dt), xm));
        double t = 0.0;
#pragma unroll
        for (int d = 0; d < 3; d++) {
            double ff = f[3 * i + d];
            if (f_add) ff = __dadd_rn(ff, f_add[3 * i + d]);
            if (subtract_mean) ff = __dsub_rn(ff, __ddiv_rn(acc[A_FSUM0 + d], (double)n));
            ff = __dadd_rn(ff, __dmul_rn(fluct_draw(seed, step, i, d, bad), beta));
            f[3 * i + d] = ff;
            const double vv = __ddiv_rn(__dadd_rn(v[3 * i + d], __ddiv_rn(__dmul_rn(__dmul_rn(0.5, dt), ff), xm)), den);
            v[3 * i + d] = vv;
            t = __dadd_rn(t, __dmul_rn(xm, __dmul_rn(vv, vv)));
        }
        mv2 = t;
    }
    if (bad) atomicOr(status, ST_RNG);   // 100 rejected polar-method attempts
    block_add<256>(mv2, acc, A_MV2, red);
}

static Masses masses(const simox_ctx* c) {
    Masses M;
    for (int s = 0; s < 5; s++) M.xm[s] = c->pot.param[s].xm;
    return M;
}

int update_masses(simox_ctx*) { return SIMOX_OK; }

int vv1(simox_ctx* c, double dt, bool reflect) {
    if (c->n == 0) return SIMOX_OK;
    {
        Launch L(c, reflect ? "vv_nve1_reflect" : "vv_nve1");
        launch_k<256, 1, vv1_body>(c, vv1_kernel, (c->n + 255) / 256, 0, c->stream, c->n, c->id, c->x, c->v, c->f, dt,
            make_double3(c->box[0], c->box[1], c->box[2]), masses(c), reflect ? 1 : 0);
    }
    c->gathered = false;
    c->list_valid = false;
    c->eam_valid = false;
    c->cells_fresh = false;
    c->in_box = !reflect;   // VV_NVE1 wraps every coordinate into [-L/2, L/2]
    return check_launch(c);
}

int vv2(simox_ctx* c, double dt, bool subtract_mean, const double* f_add) {
    memset_async(c, c->acc + A_MV2, 0, sizeof(double), c->stream);
    if (c->n == 0) return SIMOX_OK;
    {
        Launch L(c, "vv_nve2");
        launch_k<256, 1, vv2_body<false>>(c, vv2_kernel<false>, (c->n + 255) / 256, 0, c->stream, c->n, c->id, c->v,
            c->f, f_add, dt, masses(c), c->acc, subtract_mean ? 1 : 0);
    }
    return check_launch(c);
}

int nvt2_berend(simox_ctx* c, double dt, double T_given, bool subtract_mean, const double* f_add) {
    memset_async(c, c->acc + A_MV2, 0, sizeof(double) * (A_NS4 + 1 - A_MV2), c->stream);
    if (c->n == 0) return SIMOX_OK;
    {
        Launch L(c, "vv_nvt2_kick");
        launch_k<256, 1, vv2_body<true>>(c, vv2_kernel<true>, (c->n + 255) / 256, 0, c->stream, c->n, c->id, c->v,
            c->f, f_add, dt, masses(c), c->acc, subtract_mean ? 1 : 0);
    }
    {
        Launch L(c, "vv_nvt2_scale");
        launch_k<256, 1, berend_scale_body>(c, berend_scale_kernel, (c->n + 255) / 256, 0, c->stream, c->n, c->id,
            c->v, masses(c), T_given, c->acc);
    }
    return check_launch(c);
}

// VINIT's velocities; its as-written mv2 lands in acc[A_MV2]
int vinit_velocities(simox_ctx* c, unsigned long long seed, double T_given) {
    cudaMemsetAsync(c->acc + A_MV2, 0, sizeof(double) * (A_NS4 + 1 - A_MV2), c->stream);
    cudaMemsetAsync(c->acc + A_LINE0, 0, sizeof(double) * 3, c->stream);
    if (c->n == 0) return SIMOX_OK;
    const int nb = (c->n + 255) / 256;
    Launch L(c, "vinit");
    vinit_draw_kernel<<<nb, 256, 0, c->stream>>>(c->n, seed, c->v, c->acc);
    vinit_center_kernel<<<nb, 256, 0, c->stream>>>(c->n, c->id, c->v, masses(c), c->acc);
    vinit_scale_kernel<<<nb, 256, 0, c->stream>>>(c->n, c->id, c->v, masses(c), T_given, c->acc);
    return check_launch(c);
}

int nvt1_stoch(simox_ctx* c, double dt, double alpha) {
    if (c->n == 0) return SIMOX_OK;
    {
        Launch L(c, "vv_nvt1_stoch");
        vv1_stoch_kernel<<<(c->n + 255) / 256, 256, 0, c->stream>>>(
            c->n, c->id, c->x, c->v, c->f, dt, alpha, make_double3(c->box[0], c->box[1], c->box[2]), masses(c));
    }
    c->gathered = false;
    c->list_valid = false;
    c->eam_valid = false;
    c->cells_fresh = false;
    c->in_box = true;   // every coordinate wrapped into [-L/2, L/2]
    return check_launch(c);
}

int nvt2_stoch(simox_ctx* c, double dt, double alpha, double T_given, unsigned long long seed,
               unsigned long long step, bool subtract_mean, const double* f_add) {
    cudaMemsetAsync(c->acc + A_MV2, 0, sizeof(double), c->stream);
    if (c->n == 0) return SIMOX_OK;
    const double beta = std::sqrt(2.0 * alpha * T_given / dt);   // vverlet.f90:280
    {
        Launch L(c, "vv_nvt2_stoch");
        vv2_stoch_kernel<<<(c->n + 255) / 256, 256, 0, c->stream>>>(c->n, c->id, c->v, c->f, f_add, dt, alpha, beta,
                                                                    seed, step, masses(c), c->acc,
                                                                    subtract_mean ? 1 : 0, c->status);
    }
    return check_launch(c);
}

}  // namespace sx
