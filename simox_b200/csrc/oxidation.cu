// oxidation.cu -- the oxidation-mode steps of main.f90:63-84 on the device.
//
// On a charge step the reference's oxidation loop runs, between CELL_SORT and
// CTIP_SOLVER,
//   REMOVE_RIGID_MOTION (vverlet.f90:211-234): v -= mean v, z -= mean z
//                        (unit masses);
//   OXIDE_CHECK          (util.f90:152-188): a new dimer is due when the
//                        highest Al atom is above the highest of the O atoms
//                        among the last 2 N_o2 atoms (heights floored at 0), or
//                        the most positive charge among those O atoms is below
//                        q_crit (floored at -10);
//   NEW_O2               (datafmt.f90:98-139) with RANDOM_POSITION_O2
//                        (util.f90:104-148): 2 N_o2 O atoms appended at height
//                        z_new in dimers of bond length 2 A, v = (0, 0,
//                        -sqrt(3 T_given / 16)), f = 0, q = 0.
// Here all three act on the device-resident state: the only host traffic of
// a charge event is the one "due" flag, which the host needs because the
// atom count -- and so every later launch -- changes with an insertion.  The
// arrays are allocated for the context's capacity, so an insertion is an
// append, not the reference's reallocation (ADD_PTCL, datafmt.f90:84-95).
//
// REMOVE_RIGID_MOTION's sums are FP64 block sums added in a fixed order (the
// same bits every run; the reference's serial sum may differ in the last
// bit).  OXIDE_CHECK takes maxima, which no order changes.  The dimer
// positions come from the library's seeded counter-based generator, stream
// (1 << 63 | event), one counter per draw in the reference's order, so an
// insertion is reproducible; the y offset of a dimer repeats the x formula
// as written (util.f90:138).
#include "simox_internal.cuh"

#include <cmath>
#include <vector>

namespace sx {

__device__ __forceinline__ unsigned long long ox_mix64(unsigned long long z) {
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
    return z ^ (z >> 31);
}
// the uniform draw of integrate.cu (SplitMix64 output mix twice, 53 bits)
__device__ __forceinline__ double ox_uniform(unsigned long long seed, unsigned long long a, unsigned long long b) {
    const unsigned long long g = 0x9E3779B97F4A7C15ULL;
    const unsigned long long z = ox_mix64(ox_mix64(seed + g * (a + 1)) + g * (b + 1));
    return (double)(z >> 11) * (1.0 / 9007199254740992.0);
}

constexpr int RR_THREADS = 256;

// per-block sums of v (3) and z in a fixed tree order
__global__ void __launch_bounds__(RR_THREADS)
    rrm_partial_kernel(int n, const double* __restrict__ x, const double* __restrict__ v,
                       double* __restrict__ part) {
    __shared__ double s[4][RR_THREADS];
    const int i = blockIdx.x * RR_THREADS + threadIdx.x;
    const bool in = i < n;
    s[0][threadIdx.x] = in ? v[3 * i] : 0.0;
    s[1][threadIdx.x] = in ? v[3 * i + 1] : 0.0;
    s[2][threadIdx.x] = in ? v[3 * i + 2] : 0.0;
    s[3][threadIdx.x] = in ? x[3 * i + 2] : 0.0;
    __syncthreads();
    for (int h = RR_THREADS / 2; h > 0; h >>= 1) {
        if (threadIdx.x < h)
            for (int c = 0; c < 4; c++) s[c][threadIdx.x] += s[c][threadIdx.x + h];
        __syncthreads();
    }
    if (threadIdx.x < 4) part[4 * blockIdx.x + threadIdx.x] = s[threadIdx.x][0];
}

// the block sums added in block order by one thread per component; means
__global__ void rrm_mean_kernel(int nb, int n, const double* __restrict__ part, double* __restrict__ mean) {
    const int c = threadIdx.x;
    if (c >= 4) return;
    double t = 0.0;
    for (int b = 0; b < nb; b++) t += part[4 * b + c];
    mean[c] = t / (double)n;
}

__global__ void rrm_apply_kernel(int n, double* __restrict__ x, double* __restrict__ v,
                                 const double* __restrict__ mean) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    v[3 * i] = __dsub_rn(v[3 * i], mean[0]);
    v[3 * i + 1] = __dsub_rn(v[3 * i + 1], mean[1]);
    v[3 * i + 2] = __dsub_rn(v[3 * i + 2], mean[2]);
    x[3 * i + 2] = __dsub_rn(x[3 * i + 2], mean[3]);
}

// Order-preserving unsigned key of a double (negative values reversed), so
// atomicMax on keys is max on the doubles.
__device__ __forceinline__ unsigned long long dkey(double d) {
    const unsigned long long u = (unsigned long long)__double_as_longlong(d);
    return (u >> 63) ? ~u : (u | 0x8000000000000000ULL);
}
__device__ __forceinline__ double dkey_value(unsigned long long k) {
    const unsigned long long u = (k >> 63) ? (k & 0x7FFFFFFFFFFFFFFFULL) : ~k;
    return __longlong_as_double((long long)u);
}

// keys[0] = max z of Al atoms, keys[1] = max z and keys[2] = max q of the O
// atoms with index >= lo (the last 2 N_o2 atoms); keys[3] = the largest
// |x_d| - L_d/2 over all atoms and axes (> 0: an atom outside the box)
__global__ void __launch_bounds__(256)
    oxide_check_kernel(int n, int lo, const int* __restrict__ id, const double* __restrict__ x,
                       const double* __restrict__ q, double3 hbox, unsigned long long* __restrict__ keys) {
    unsigned long long m = 0ull, oh = 0ull, qm = 0ull, ob = 0ull;   // key 0: below every double
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const int s = id[i];
        const double z = x[3 * i + 2];
        if (s == 1) m = max(m, dkey(z));
        if (s == 4 && i >= lo) {
            oh = max(oh, dkey(z));
            qm = max(qm, dkey(q[i]));
        }
        const double out = fmax(fmax(fabs(x[3 * i]) - hbox.x, fabs(x[3 * i + 1]) - hbox.y), fabs(z) - hbox.z);
        ob = max(ob, dkey(out));
    }
    for (int o = 16; o > 0; o >>= 1) {
        m = max(m, __shfl_xor_sync(0xffffffffu, m, o));
        oh = max(oh, __shfl_xor_sync(0xffffffffu, oh, o));
        qm = max(qm, __shfl_xor_sync(0xffffffffu, qm, o));
        ob = max(ob, __shfl_xor_sync(0xffffffffu, ob, o));
    }
    if ((threadIdx.x & 31) == 0) {
        if (m) atomicMax(keys, m);
        if (oh) atomicMax(keys + 1, oh);
        if (qm) atomicMax(keys + 2, qm);
        if (ob) atomicMax(keys + 3, ob);
    }
}

// due[0]: a dimer is due; due[1]: every atom lies inside the box
__global__ void oxide_decide_kernel(const unsigned long long* __restrict__ keys, double q_crit, int* __restrict__ due) {
    // the reference's floors: heights start at 0, the charge at -10
    const double m_height = keys[0] ? fmax(dkey_value(keys[0]), 0.0) : 0.0;
    const double o_height = keys[1] ? fmax(dkey_value(keys[1]), 0.0) : 0.0;
    const double q_max = keys[2] ? fmax(dkey_value(keys[2]), -10.0) : -10.0;
    due[0] = ((m_height + 0.0) > o_height || q_max < q_crit) ? 1 : 0;
    due[1] = (keys[3] == 0ull || dkey_value(keys[3]) <= 0.0) ? 1 : 0;
}

// RANDOM_POSITION_O2 (util.f90:104-148) in one thread: the rejection loop is
// sequential in the reference's draw order.  Writes 2 n_o2 positions to xx,
// or sets *fail (no room after 100,000 tries for one dimer).
__global__ void random_position_o2_kernel(int n_o2, double z_new, double Lx, double Ly, unsigned long long seed,
                                          unsigned long long event, double* __restrict__ cx,
                                          double* __restrict__ xx, int* __restrict__ fail) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    const double L0 = 2.0;
    const double rc = sqrt(Lx * Ly / (double)n_o2) * 0.5;
    const double rc2 = rc * rc;
    const unsigned long long a = (1ULL << 63) | event;
    unsigned long long k = 0;
    cx[0] = (ox_uniform(seed, a, k++) - 0.5) * Lx;
    cx[1] = (ox_uniform(seed, a, k++) - 0.5) * Ly;
    for (int i = 1; i < n_o2; i++) {
        bool placed = false;
        for (int t = 0; t < 100000 && !placed; t++) {
            cx[3 * i] = (ox_uniform(seed, a, k++) - 0.5) * Lx;
            cx[3 * i + 1] = (ox_uniform(seed, a, k++) - 0.5) * Ly;
            placed = true;
            for (int j = 0; j < i; j++) {
                const double dx = __dsub_rn(cx[3 * i], cx[3 * j]), dy = __dsub_rn(cx[3 * i + 1], cx[3 * j + 1]);
                if (__dadd_rn(__dmul_rn(dx, dx), __dmul_rn(dy, dy)) < rc2) placed = false;   // no FMA: the oracle's test
            }
        }
        if (!placed) {
            *fail = 1;
            return;
        }
    }
    for (int i = 0; i < n_o2; i++) {
        cx[3 * i + 2] = z_new;
        const double phi = ox_uniform(seed, a, k++) * SX_PI * 2.0;
        const double theta = ox_uniform(seed, a, k++) * SX_PI;
        const double st = sin(theta), cp = cos(phi);
        const double d[3] = {L0 * st * cp, L0 * st * cp, L0 * cos(theta)};   // y as written (util.f90:138)
        for (int c = 0; c < 3; c++) {
            xx[3 * (2 * i) + c] = __dadd_rn(d[c], cx[3 * i + c]);
            xx[3 * (2 * i + 1) + c] = __dadd_rn(-d[c], cx[3 * i + c]);
        }
    }
}

// NEW_O2's new atoms (datafmt.f90:118-135) at indices n0 .. n0 + m - 1
__global__ void append_o2_kernel(int n0, int m, const double* __restrict__ xx, double vz, int* __restrict__ id,
                                 double* __restrict__ x, double* __restrict__ v, double* __restrict__ f,
                                 double* __restrict__ q, const int* __restrict__ fail) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= m || *fail) return;
    const int i = n0 + k;
    id[i] = 4;
    for (int c = 0; c < 3; c++) {
        x[3 * i + c] = xx[3 * k + c];
        v[3 * i + c] = 0.0;
        f[3 * i + c] = 0.0;
    }
    v[3 * i + 2] = -vz;
    q[i] = 0.0;
}

// The moved atoms invalidate every copy in pair order and the neighbour list.
static void positions_moved(simox_ctx* c) {
    c->gathered = false;
    c->list_valid = false;
    c->eam_valid = false;
    c->cells_fresh = false;
    c->rho_ready = false;
}

int remove_rigid_motion(simox_ctx* c) {
    const int n = c->n;
    if (n <= 0) return SIMOX_OK;
    const int nb = (n + RR_THREADS - 1) / RR_THREADS;
    // scratch: the block sums in the charge solver's work vector (free
    // between solves), the means in its scalar slots
    double* part = c->Ap;
    double* mean = c->line + 56;
    if ((size_t)4 * nb > (size_t)c->cap) return SIMOX_E_CAPACITY;
    {
        Launch L(c, "remove_rigid_motion");
        rrm_partial_kernel<<<nb, RR_THREADS, 0, c->stream>>>(n, c->x, c->v, part);
        rrm_mean_kernel<<<1, 32, 0, c->stream>>>(nb, n, part, mean);
        rrm_apply_kernel<<<nb, RR_THREADS, 0, c->stream>>>(n, c->x, c->v, mean);
    }
    positions_moved(c);
    return check_launch(c);
}

int oxide_check(simox_ctx* c, int n_o2, double q_crit, int* due) {
    const int n = c->n;
    unsigned long long* keys = reinterpret_cast<unsigned long long*>(c->line + 48);
    int* d_due = reinterpret_cast<int*>(c->line + 53);
    cudaMemsetAsync(keys, 0, 4 * sizeof(unsigned long long), c->stream);
    {
        Launch L(c, "oxide_check");
        if (n > 0) {
            const int lo = n - 2 * n_o2;
            const int g = std::min((n + 255) / 256, num_sms(c) * 4);
            oxide_check_kernel<<<g, 256, 0, c->stream>>>(n, lo, c->id, c->x, c->q,
                                                         make_double3(c->hbox[0], c->hbox[1], c->hbox[2]), keys);
        }
        oxide_decide_kernel<<<1, 1, 0, c->stream>>>(keys, q_crit, d_due);
    }
    if (int st = check_launch(c)) return st;
    int h[2] = {0, 1};
    cudaMemcpyAsync(h, d_due, 2 * sizeof(int), cudaMemcpyDeviceToHost, c->stream);
    if (int st = cuda_status(cudaStreamSynchronize(c->stream))) return st;
    *due = h[0];
    c->in_box = h[1] != 0;   // the skin list's pair set equals the reference's only inside the box
    return SIMOX_OK;
}

int new_o2(simox_ctx* c, int n_o2, double z_new, double T_given, unsigned long long seed,
           unsigned long long event) {
    if (n_o2 <= 0) return SIMOX_OK;
    const int m = 2 * n_o2;
    if (c->n + m > c->cap) return SIMOX_E_CAPACITY;
    // "=== Too many new oxygens ===" (util.f90:118): the dimers' spacing
    // would be below the bond length
    if (std::sqrt(c->box[0] * c->box[1] / (double)n_o2) * 0.5 < 2.0) return SIMOX_E_ARG;
    // scratch: centres and positions in the charge solver's work vectors
    if ((size_t)3 * m > (size_t)c->cap) return SIMOX_E_CAPACITY;
    double* cx = c->g;
    double* xx = c->pv;
    int* fail = reinterpret_cast<int*>(c->line + 55);
    const int n0 = c->n;
    cudaMemsetAsync(fail, 0, sizeof(int), c->stream);
    {
        Launch L(c, "new_o2");
        random_position_o2_kernel<<<1, 1, 0, c->stream>>>(n_o2, z_new, c->box[0], c->box[1], seed, event, cx, xx,
                                                          fail);
        append_o2_kernel<<<(m + 127) / 128, 128, 0, c->stream>>>(n0, m, xx, std::sqrt(T_given * 3.0 / 16.0), c->id,
                                                                 c->x, c->v, c->f, c->q, fail);
    }
    if (int st = check_launch(c)) return st;
    // the host learns the outcome and whether the new atoms lie in the box
    std::vector<double> hx((size_t)3 * m);
    int h_fail = 0;
    cudaMemcpyAsync(hx.data(), xx, sizeof(double) * 3 * m, cudaMemcpyDeviceToHost, c->stream);
    cudaMemcpyAsync(&h_fail, fail, sizeof(int), cudaMemcpyDeviceToHost, c->stream);
    if (int st = cuda_status(cudaStreamSynchronize(c->stream))) return st;
    if (h_fail) return SIMOX_E_ARG;
    bool inb = c->in_box;
    for (int k = 0; k < m && inb; k++)
        for (int d = 0; d < 3; d++) inb = inb && std::fabs(hx[3 * k + d]) <= c->hbox[d];
    c->in_box = inb;
    c->n = n0 + m;
    c->cells_valid = false;
    c->skin_valid = false;
    positions_moved(c);
    drop_graphs(c);
    return SIMOX_OK;
}

}  // namespace sx

using namespace sx;

// REMOVE_RIGID_MOTION vverlet.f90:211-234
extern "C" int simox_remove_rigid_motion(simox_ctx* c) {
    if (!c) return SIMOX_E_ARG;
    cudaSetDevice(c->device);
    const int st = remove_rigid_motion(c);
    return st ? st : cuda_status(cudaStreamSynchronize(c->stream));
}

// OXIDE_CHECK util.f90:152-188
extern "C" int simox_oxide_check(simox_ctx* c, int n_o2, double q_crit, int* due) {
    if (!c || !due || n_o2 < 0) return SIMOX_E_ARG;
    cudaSetDevice(c->device);
    return oxide_check(c, n_o2, q_crit, due);
}

// NEW_O2 datafmt.f90:98-139 with RANDOM_POSITION_O2 util.f90:104-148
extern "C" int simox_new_o2(simox_ctx* c, int n_o2, double z_new, double T_given, unsigned long long seed,
                            unsigned long long event) {
    if (!c || n_o2 < 0 || !c->have_ids) return SIMOX_E_ARG;
    cudaSetDevice(c->device);
    return new_o2(c, n_o2, z_new, T_given, seed, event);
}
