// integrate.cu -- velocity-Verlet kernels of vverlet.f90.
//
// Each kernel reproduces the reference's FP64 operation order with explicit
// round-to-nearest intrinsics (no FMA contraction), so given the same forces
// the positions and velocities are bit-identical to the Fortran statements:
//   VV_NVE1         vverlet.f90:74-96    v += 0.5 dt f/m; x += dt v; x -= L DNINT(x/L)
//   VV_NVE1_REFLECT vverlet.f90:100-129  same, z reflected at +L/2 instead of wrapped
//   VV_NVE2         vverlet.f90:132-157  v += 0.5 dt f/m; mv2 = sum m v^2
//   VV_NVT2_BEREND  vverlet.f90:160-208  half kick, per-species T, v *= lambda_s
// The second half kick optionally first removes the mean PME force
// (force.f90:457-460), f = f - Fsum/N, and stores the final force.
#include "simox_internal.cuh"

namespace sx {

struct Masses { double xm[5]; };

__device__ __forceinline__ double half_kick(double v, double f, double dt, double xm) {
    return __dadd_rn(v, __ddiv_rn(__dmul_rn(__dmul_rn(0.5, dt), f), xm));
}

__global__ void vv1_kernel(int n, const int* __restrict__ id, double* __restrict__ x, double* __restrict__ v,
                           const double* __restrict__ f, double dt, double3 box, Masses M, int reflect) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
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

// second half kick (+ optional mean-force removal); mv2 and per-species sums
template <bool BEREND>
__global__ void __launch_bounds__(256)
    vv2_kernel(int n, const int* __restrict__ id, double* __restrict__ v, double* __restrict__ f,
               const double* __restrict__ f_add, double dt, Masses M, double* __restrict__ acc, int subtract_mean) {
    __shared__ double red[256 / 32];
    double mv2 = 0.0;
    double ms[5] = {0, 0, 0, 0, 0};
    double ns[5] = {0, 0, 0, 0, 0};
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
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

// Berendsen rescale (vverlet.f90:188-205)
__global__ void __launch_bounds__(256)
    berend_scale_kernel(int n, const int* __restrict__ id, double* __restrict__ v, Masses M, double T_given,
                        double* __restrict__ acc) {
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
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
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
        vv1_kernel<<<(c->n + 255) / 256, 256, 0, c->stream>>>(c->n, c->id, c->x, c->v, c->f, dt,
                                                              make_double3(c->box[0], c->box[1], c->box[2]), masses(c),
                                                              reflect ? 1 : 0);
    }
    c->gathered = false;
    c->list_valid = false;
    c->eam_valid = false;
    c->cells_fresh = false;
    c->in_box = !reflect;   // VV_NVE1 wraps every coordinate into [-L/2, L/2]
    return check_launch(c);
}

int vv2(simox_ctx* c, double dt, bool subtract_mean, const double* f_add) {
    cudaMemsetAsync(c->acc + A_MV2, 0, sizeof(double), c->stream);
    if (c->n == 0) return SIMOX_OK;
    {
        Launch L(c, "vv_nve2");
        vv2_kernel<false><<<(c->n + 255) / 256, 256, 0, c->stream>>>(c->n, c->id, c->v, c->f, f_add, dt, masses(c),
                                                                     c->acc, subtract_mean ? 1 : 0);
    }
    return check_launch(c);
}

int nvt2_berend(simox_ctx* c, double dt, double T_given, bool subtract_mean, const double* f_add) {
    cudaMemsetAsync(c->acc + A_MV2, 0, sizeof(double) * (A_NS4 + 1 - A_MV2), c->stream);
    if (c->n == 0) return SIMOX_OK;
    {
        Launch L(c, "vv_nvt2_kick");
        vv2_kernel<true><<<(c->n + 255) / 256, 256, 0, c->stream>>>(c->n, c->id, c->v, c->f, f_add, dt, masses(c),
                                                                    c->acc, subtract_mean ? 1 : 0);
    }
    {
        Launch L(c, "vv_nvt2_scale");
        berend_scale_kernel<<<(c->n + 255) / 256, 256, 0, c->stream>>>(c->n, c->id, c->v, masses(c), T_given, c->acc);
    }
    return check_launch(c);
}

}  // namespace sx
