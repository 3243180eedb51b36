// cells.cu -- CELL_HIERARCHY / CELL_SORT (cellsort.f90) and the neighbour-list
// build of the pair loops (force.f90:41-58,146-162; ctip.f90:64-80,116-130).
//
// Binning is a counting sort: cell id per atom with the reference's FP64
// arithmetic (xx = x + L/2; INT(xx/Lcell); MOD(id + Ncell, Ncell)), an atomic
// histogram, an exclusive scan, a scatter and a per-cell rank sort that puts
// each cell's atoms in ascending original index -- the order CELL_SORT's
// serial loop appends them (cellsort.f90:68-76).  Membership and order are
// therefore bit-exact.
//
// The neighbour list is a full list (each pair in both rows) in cell-sorted
// index space.  One CTA per home cell stages the 27 stencil cells' atoms in
// shared memory as FP32 offsets from the home-cell centre; each thread owns a
// home atom and tests every staged candidate with an FP32 distance.  Pairs
// within a relative band of 4e-5 around Rcut^2 are re-tested with the
// reference's exact FP64 expression (dx - L*DNINT(dx/L), r2 summed without
// FMA), so list membership equals the reference's r2 < Rcut2 test.  Rows are
// grouped by partner species (metals from the front, oxygen from the back).
#include "simox_internal.cuh"

#include <algorithm>
#include <cstring>

namespace sx {

// list build: one thread per home atom of a cell (a skin cell of the 128k
// corundum holds ~180 atoms: with 128 threads a third of them walked two
// home atoms one after the other)
constexpr int LB_THREADS = 256;
constexpr int LB_TILE = 1024;

// ---------------------------------------------------------------------------
// CELL_HIERARCHY cellsort.f90:3-36 (host): 13-cell half stencil, 1-based ids
static int id_cell(const int nc[3], int i, int j, int k) {
    int l = (i - 1 + nc[0]) % nc[0];
    int m = (j - 1 + nc[1]) % nc[1];
    int n = (k - 1 + nc[2]) % nc[2];
    return l + m * nc[0] + n * nc[0] * nc[1] + 1;
}

int list_prepare(simox_ctx* c);

int build_cell_tables(simox_ctx* c) {
    const int* nc = c->nc;
    const int ncell = c->ncell;
    std::vector<int>& P = c->h_pair13;
    P.assign((size_t)ncell * 13, 0);
    static const int off[13][3] = {{-1, -1, -1}, {0, -1, -1}, {1, -1, -1}, {-1, 0, -1}, {0, 0, -1},
                                   {1, 0, -1},   {-1, 1, -1}, {0, 1, -1},  {1, 1, -1},  {-1, -1, 0},
                                   {0, -1, 0},   {1, -1, 0},  {-1, 0, 0}};
    for (int i = 1; i <= nc[0]; i++)
        for (int j = 1; j <= nc[1]; j++)
            for (int k = 1; k <= nc[2]; k++) {
                int id = id_cell(nc, i, j, k);
                for (int n = 0; n < 13; n++)
                    P[(size_t)(id - 1) * 13 + n] = id_cell(nc, i + off[n][0], j + off[n][1], k + off[n][2]);
            }
    // Full stencil with multiplicity: self, the 13 forward cells, and every
    // cell whose forward list names this one.  dir: 0 self, 1 forward
    // (this atom is the reference's "i"), 2 reverse.
    std::vector<int> E((size_t)ncell * kEntries, 0);
    std::vector<int> fill(ncell, 0);
    for (int cc = 0; cc < ncell; cc++) {
        E[(size_t)cc * kEntries + fill[cc]++] = cc;
        for (int n = 0; n < 13; n++) E[(size_t)cc * kEntries + fill[cc]++] = (P[(size_t)cc * 13 + n] - 1) | (1 << 28);
    }
    for (int cc = 0; cc < ncell; cc++)
        for (int n = 0; n < 13; n++) {
            int t = P[(size_t)cc * 13 + n] - 1;
            if (fill[t] >= kEntries) return SIMOX_E_CELL_TOO_SMALL;
            E[(size_t)t * kEntries + fill[t]++] = cc | (2 << 28);
        }
    for (int cc = 0; cc < ncell; cc++)
        if (fill[cc] != kEntries) return SIMOX_E_CELL_TOO_SMALL;
    if (int st = list_prepare(c)) return st;
    cudaError_t e1 = cudaMemcpyAsync(c->pair13, P.data(), P.size() * sizeof(int), cudaMemcpyHostToDevice, c->stream);
    cudaError_t e2 = cudaMemcpyAsync(c->entries, E.data(), E.size() * sizeof(int), cudaMemcpyHostToDevice, c->stream);
    if (e1 != cudaSuccess || e2 != cudaSuccess) return SIMOX_E_CUDA;
    return cuda_status(cudaStreamSynchronize(c->stream));
}

// ---------------------------------------------------------------------------
// CELL_SORT kernels
__device__ __forceinline__ void bin_atoms_body(Blk B, int n, const double* __restrict__ x, double3 hbox, double3 lc,
                                               int3 nc, int* __restrict__ cell_of, int* __restrict__ cell_xyz,
                                               int* __restrict__ count, int* __restrict__ status) {
    int i = B.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    int id[3];
    const double hb[3] = {hbox.x, hbox.y, hbox.z};
    const double l[3] = {lc.x, lc.y, lc.z};
    const int m[3] = {nc.x, nc.y, nc.z};
    bool bad = false;
    for (int d = 0; d < 3; d++) {
        double xx = __dadd_rn(x[3 * i + d], hb[d]);     // xx = x + hbox   cellsort.f90:69
        double t = __ddiv_rn(xx, l[d]);                 // xx/Lcell        cellsort.f90:70
        if (!(fabs(t) < 1.0e9)) { bad = true; id[d] = 0; continue; }
        int v = __double2int_rz(t);                     // INT(): toward zero
        v = (v + m[d]) % m[d];                          // MOD(id+Ncell, Ncell) cellsort.f90:71
        if (v < 0) { bad = true; v = 0; }
        id[d] = v;
    }
    if (bad) atomicOr(status, ST_POSITION);
    int cell = id[0] + id[1] * m[0] + id[2] * m[0] * m[1];
    cell_of[i] = cell;
    cell_xyz[i] = id[0] | (id[1] << 10) | (id[2] << 20);   // Ncell <= 1024 per axis (checked at set-up)
    atomicAdd(count + cell, 1);
}
__global__ void bin_atoms_kernel(int n, const double* __restrict__ x, double3 hbox, double3 lc, int3 nc,
                                 int* __restrict__ cell_of, int* __restrict__ cell_xyz, int* __restrict__ count,
                                 int* __restrict__ status) {
    bin_atoms_body(own_blk(), n, x, hbox, lc, nc, cell_of, cell_xyz, count, status);
}

// cond: nullptr, or a device flag that must be non-zero for the kernel to run
// (the skin-list rebuild is decided on the device, without a host round trip)
__device__ __forceinline__ void scan_cells_body(Blk B, const int* __restrict__ count, int* __restrict__ start,
                                                int* __restrict__ fill, int ncell, int npt_max,
                                                int* __restrict__ status, const int* __restrict__ cond) {
    if (cond && *cond == 0) return;
    __shared__ int sm[1024];
    __shared__ int carry;
    const int t = threadIdx.x;
    if (t == 0) carry = 0;
    __syncthreads();
    for (int base = 0; base < ncell; base += 1024) {
        int v = base + t < ncell ? count[base + t] : 0;
        if (v > npt_max) atomicOr(status, ST_CELL_OVERFLOW);
        sm[t] = v;
        __syncthreads();
        for (int off = 1; off < 1024; off <<= 1) {
            int add = t >= off ? sm[t - off] : 0;
            __syncthreads();
            sm[t] += add;
            __syncthreads();
        }
        int excl = sm[t] - v + carry;
        if (base + t < ncell) { start[base + t] = excl; fill[base + t] = excl; }
        __syncthreads();
        if (t == 1023) carry += sm[1023];
        __syncthreads();
    }
    if (t == 0) start[ncell] = carry;
}
__global__ void scan_cells_kernel(const int* __restrict__ count, int* __restrict__ start, int* __restrict__ fill,
                                  int ncell, int npt_max, int* __restrict__ status, const int* __restrict__ cond) {
    scan_cells_body(own_blk(), count, start, fill, ncell, npt_max, status, cond);
}

__device__ __forceinline__ void scatter_atoms_body(Blk B, int n, const int* __restrict__ cell_of,
                                                   int* __restrict__ fill, int* __restrict__ sorted,
                                                   const int* __restrict__ cond) {
    if (cond && *cond == 0) return;
    int i = B.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    int slot = atomicAdd(fill + cell_of[i], 1);
    sorted[slot] = i;
}
__global__ void scatter_atoms_kernel(int n, const int* __restrict__ cell_of, int* __restrict__ fill,
                                     int* __restrict__ sorted, const int* __restrict__ cond) {
    scatter_atoms_body(own_blk(), n, cell_of, fill, sorted, cond);
}

// Rank sort inside each cell: ascending original index (= CELL_SORT order).
__device__ __forceinline__ void cell_rank_sort_body(Blk B, const int* __restrict__ start, int* __restrict__ sorted,
                                                    int npt_max, const int* __restrict__ cond) {
    if (cond && *cond == 0) return;
    extern __shared__ int buf[];
    const int cc = B.x;
    const int s0 = start[cc], n = start[cc + 1] - s0;
    if (n <= 1 || n > npt_max) return;
    for (int k = threadIdx.x; k < n; k += blockDim.x) buf[k] = sorted[s0 + k];
    __syncthreads();
    for (int k = threadIdx.x; k < n; k += blockDim.x) {
        int v = buf[k], rank = 0;
        for (int m = 0; m < n; m++) rank += buf[m] < v;
        sorted[s0 + rank] = v;
    }
}
__global__ void cell_rank_sort_kernel(const int* __restrict__ start, int* __restrict__ sorted, int npt_max,
                                      const int* __restrict__ cond) {
    cell_rank_sort_body(own_blk(), start, sorted, npt_max, cond);
}

int cell_sort(simox_ctx* c) {
    if (!c->have_ids) return SIMOX_E_STATE;
    const int n = c->n;
    memset_async(c, c->cell_count, 0, sizeof(int) * c->ncell, c->stream);
    if (n > 0) {
        Launch L(c, "cell_bin");
        launch_k<256, 1, bin_atoms_body>(c, bin_atoms_kernel, (n + 255) / 256, 0, c->stream, n, c->x,
            make_double3(c->hbox[0], c->hbox[1], c->hbox[2]), make_double3(c->lc[0], c->lc[1], c->lc[2]),
            make_int3(c->nc[0], c->nc[1], c->nc[2]), c->cell_of, c->cell_xyz, c->cell_count, c->status);
    }
    {
        Launch L(c, "cell_scan");
        launch_k<1024, 1, scan_cells_body>(c, scan_cells_kernel, 1, 0, c->stream, c->cell_count, c->cell_start,
            c->cell_fill, c->ncell, c->npt_max, c->status, nullptr);
    }
    int st = check_launch(c);
    if (st) return st;
    c->cells_valid = true;
    c->cells_fresh = true;
    c->cells_listed = false;   // the link lists themselves are filled when something reads them
    c->gathered = false;
    c->list_valid = false;
    return SIMOX_OK;
}

// The reference cells' link lists (sorted: atoms cell by cell, ascending
// within a cell, cellsort.f90:69-78) of the last CELL_SORT.  In skin mode the
// pair kernels run in the skin order and only simox_get_cells reads them, so
// CELL_SORT leaves them to this call (the binning, the counts and the
// over-full-cell check run every time).
int ensure_cell_lists(simox_ctx* c) {
    if (!c->cells_valid) return SIMOX_E_STATE;
    if (c->cells_listed) return SIMOX_OK;
    const int n = c->n;
    if (n > 0) {
        Launch L(c, "cell_scatter");
        launch_k<256, 1, scatter_atoms_body>(c, scatter_atoms_kernel, (n + 255) / 256, 0, c->stream, n, c->cell_of,
            c->cell_fill, c->sorted, nullptr);
    }
    {
        Launch L(c, "cell_order");
        launch_k<128, 1, cell_rank_sort_body>(c, cell_rank_sort_kernel, c->ncell, sizeof(int) * c->npt_max, c->stream,
            c->cell_start, c->sorted, c->npt_max, nullptr);
    }
    int st = check_launch(c);
    if (st) return st;
    c->cells_listed = true;
    return SIMOX_OK;
}

// ---------------------------------------------------------------------------
// gather original-order state into cell order
// Skin-mode records of each atom (pair order): its offset from the centre
// of the skin cell it was binned into at the last rebuild (minimum image,
// FP32), with w = reference cell (9 bits per axis) | species << 27 for the
// list filter and w = charge for the force pass.
// For a skin pair (X, Y) with stencil offset o, x_Y - x_X = off_Y - off_X +
// o * Lcs exactly while both atoms stay within skin/2 of their rebuild
// positions.
struct RecParams {
    double3 box, ibox, origin, lc;
    int3 ncs;
};

__device__ __forceinline__ void gather_sorted_body(Blk B, int n, const int* __restrict__ sorted,
                                                   const double* __restrict__ x, const double* __restrict__ q,
                                                   const int* __restrict__ id, double4* __restrict__ xq,
                                                   int* __restrict__ ts, const int* __restrict__ cell_xyz,
                                                   const int* __restrict__ cs_cell_of, const RecParams& R,
                                                   float4* __restrict__ rec, float4* __restrict__ frec,
                                                   double4* __restrict__ xo) {
    int k = B.x * blockDim.x + threadIdx.x;
    if (k >= n) return;
    int o = sorted[k];
    const double x0 = x[3 * o], x1 = x[3 * o + 1], x2 = x[3 * o + 2];
    const int t = id[o] - 1;
    xq[k] = make_double4(x0, x1, x2, q[o]);
    ts[k] = t;
    if (rec) {
        const int cs = cs_cell_of[o];
        const int ci = cs % R.ncs.x, cj = (cs / R.ncs.x) % R.ncs.y, ck = cs / (R.ncs.x * R.ncs.y);
        double ox = x0 - (R.origin.x + (ci + 0.5) * R.lc.x);
        double oy = x1 - (R.origin.y + (cj + 0.5) * R.lc.y);
        double oz = x2 - (R.origin.z + (ck + 0.5) * R.lc.z);
        ox -= R.box.x * rint(ox * R.ibox.x);
        oy -= R.box.y * rint(oy * R.ibox.y);
        oz -= R.box.z * rint(oz * R.ibox.z);
        const unsigned cx = (unsigned)cell_xyz[o];
        const unsigned sp = (unsigned)t < (unsigned)kSpecies ? (unsigned)t : 7u;
        const unsigned w = (cx & 511u) | (((cx >> 10) & 511u) << 9) | (((cx >> 20) & 511u) << 18) | (sp << 27);
        rec[k] = make_float4((float)ox, (float)oy, (float)oz, __uint_as_float(w));
        frec[k] = make_float4((float)ox, (float)oy, (float)oz, (float)q[o]);
        xo[k] = make_double4(ox, oy, oz, q[o]);
    }
}
__global__ void gather_sorted_kernel(int n, const int* __restrict__ sorted, const double* __restrict__ x,
                                     const double* __restrict__ q, const int* __restrict__ id,
                                     double4* __restrict__ xq, int* __restrict__ ts, const int* __restrict__ cell_xyz,
                                     const int* __restrict__ cs_cell_of, const __grid_constant__ RecParams R,
                                     float4* __restrict__ rec, float4* __restrict__ frec, double4* __restrict__ xo) {
    gather_sorted_body(own_blk(), n, sorted, x, q, id, xq, ts, cell_xyz, cs_cell_of, R, rec, frec, xo);
}

int gather_sorted(simox_ctx* c) {
    if (!c->cells_valid) return SIMOX_E_STATE;
    if (c->n > 0) {
        Launch L(c, "gather_sorted");
        RecParams R;
        R.box = make_double3(c->box[0], c->box[1], c->box[2]);
        R.ibox = make_double3(c->inv_box[0], c->inv_box[1], c->inv_box[2]);
        R.origin = make_double3(-c->hbox[0], -c->hbox[1], -c->hbox[2]);
        R.lc = make_double3(c->lcs[0], c->lcs[1], c->lcs[2]);
        R.ncs = make_int3(c->ncs[0], c->ncs[1], c->ncs[2]);
        const bool skin = c->pair_order == c->perm && c->skin_mode;
        launch_k<256, 1, gather_sorted_body>(c, gather_sorted_kernel, (c->n + 255) / 256, 0, c->stream, c->n,
            c->pair_order, c->x, c->q, c->id, c->xq_s, c->t_s, c->cell_xyz, c->cs_cell_of, R,
            skin ? c->rec_s : nullptr, c->frec_s, c->xo_s);
    }
    c->gathered = true;
    c->rho_ready = false;
    return SIMOX_OK;
}

// ---------------------------------------------------------------------------
// neighbour list
//
// Rows are grouped by partner species: metal partners fill a row from the
// front, oxygen partners from the back (row[cap-1], row[cap-2], ...), and
// nn[i] = (n_metal, n_oxygen).  A warp looping over one group therefore sees
// one partner species, so the pair kernels run species-specialised code
// without divergence.
struct LBParams {
    double3 box, ibox, origin, lc;
    int3 nc;
    double rcut2;
    float r2lo, r2hi, hlx, hly, hlz;
    int cap, npt_max;
    int skin;   // skin list: entries carry the stencil code instead of "is i"
    int half;   // skin list: keep a pair once (forward stencil positions, or the own cell and j > h)
};

// half skin list: partner j of home atom h in stencil position e is kept by h
// when e is one of the 13 forward positions, or e is h's own cell and j > h
__device__ __forceinline__ bool half_keep(const LBParams& P, unsigned tag, int j, int h) {
    const int e = (int)(tag >> kSkinCodeShift);
    return !P.half || e > 13 || (e == 13 && j > h);
}

// reference r2 (force.f90:51-53): rx = dx - box*DNINT(dx/box), no FMA
__device__ __forceinline__ double exact_r2(double4 a, double4 b, double3 box) {
    double dx = __dsub_rn(a.x, b.x), dy = __dsub_rn(a.y, b.y), dz = __dsub_rn(a.z, b.z);
    dx = __dsub_rn(dx, __dmul_rn(box.x, round(__ddiv_rn(dx, box.x))));
    dy = __dsub_rn(dy, __dmul_rn(box.y, round(__ddiv_rn(dy, box.y))));
    dz = __dsub_rn(dz, __dmul_rn(box.z, round(__ddiv_rn(dz, box.z))));
    return __dadd_rn(__dadd_rn(__dmul_rn(dx, dx), __dmul_rn(dy, dy)), __dmul_rn(dz, dz));
}

__device__ __forceinline__ void list_append(unsigned* row, int2& my, int cap, unsigned val, int sp) {
    const int used = my.x + my.y;
    if (sp == 3) {
        if (used < cap) row[cap - 1 - my.y] = val;
        my.y++;
    } else {
        if (used < cap) row[my.x] = val;
        my.x++;
    }
}

// FAST (every Ncell >= 3 and L/2 > Rcut + Lcell/2): candidates are staged as
// FP32 offsets from the home-cell centre, already minimum-imaged with respect
// to that centre; for a home atom inside its cell that offset difference is
// the pair's minimum image, so the inner loop is three subtractions and a
// squared norm.  Pairs within 4e-5 of Rcut^2, home atoms outside their cell
// and the generic (multi-image) path use the reference's exact FP64 r2.
template <bool FAST>
__device__ __forceinline__ void build_list_body(Blk B, const int* __restrict__ cell_start,
                                                const int* __restrict__ entries, const double4* __restrict__ xq,
                                                const int* __restrict__ ts, unsigned* __restrict__ nbr,
                                                int2* __restrict__ nn, const LBParams& P, int* __restrict__ status,
                                                int* __restrict__ nn_max, unsigned long long* __restrict__ nn_tot,
                                                const int* __restrict__ cond) {
    if (cond && *cond == 0) return;
    extern __shared__ __align__(16) unsigned char smem[];
    float4* cpos = reinterpret_cast<float4*>(smem);
    unsigned* ctag = reinterpret_cast<unsigned*>(cpos + LB_TILE);
    int2* cnt = reinterpret_cast<int2*>(ctag + LB_TILE);
    __shared__ int es0[kEntries], edir[kEntries], epre[kEntries + 1];

    const int cc = B.x;
    const int h0 = cell_start[cc], nh = cell_start[cc + 1] - h0;
    if (nh <= 0) return;
    const int tid = threadIdx.x;
    if (nh > P.npt_max) {   // over-full cell: CELL_SORT already flagged it; touch nothing
        if (tid == 0) atomicOr(status, ST_CELL_OVERFLOW);
        return;
    }
    if (tid < kEntries) {
        int ent = entries[cc * kEntries + tid];
        int ce = ent & 0x0fffffff;
        es0[tid] = cell_start[ce];
        // a half skin list keeps nothing from the 13 backward stencil cells
        // (half_keep): they are not scanned
        epre[tid + 1] = (P.skin && P.half && tid < 13) ? 0 : cell_start[ce + 1] - cell_start[ce];
        edir[tid] = ent >> 28;
    }
    for (int k = tid; k < nh; k += blockDim.x) cnt[k] = make_int2(0, 0);
    __syncthreads();
    if (tid == 0) {
        epre[0] = 0;
        for (int e = 0; e < kEntries; e++) epre[e + 1] += epre[e];
    }
    __syncthreads();
    const int T = epre[kEntries];
    const int cz = cc / (P.nc.x * P.nc.y), cy = (cc / P.nc.x) % P.nc.y, cx = cc % P.nc.x;
    const double cen_x = P.origin.x + (cx + 0.5) * P.lc.x;
    const double cen_y = P.origin.y + (cy + 0.5) * P.lc.y;
    const double cen_z = P.origin.z + (cz + 0.5) * P.lc.z;

    for (int t0 = 0; t0 < T; t0 += LB_TILE) {
        const int tn = min(LB_TILE, T - t0);
        __syncthreads();
        for (int k = tid; k < tn; k += blockDim.x) {
            int g = t0 + k, e = 0;
            while (epre[e + 1] <= g) e++;
            const int j = es0[e] + (g - epre[e]);
            const double4 p = xq[j];
            double rx = p.x - cen_x, ry = p.y - cen_y, rz = p.z - cen_z;
            rx -= P.box.x * rint(rx * P.ibox.x);
            ry -= P.box.y * rint(ry * P.ibox.y);
            rz -= P.box.z * rint(rz * P.ibox.z);
            cpos[k] = make_float4((float)rx, (float)ry, (float)rz, __int_as_float(ts[j]));
            // exact list: j | dir << 30; skin list: j | stencil position << 26
            ctag[k] = P.skin ? (unsigned)j | ((unsigned)e << kSkinCodeShift) : (unsigned)j | ((unsigned)edir[e] << 30);
        }
        __syncthreads();
        for (int hl = tid; hl < nh; hl += blockDim.x) {
            const int h = h0 + hl;
            const double4 xh = xq[h];
            const float hx = (float)(xh.x - cen_x), hy = (float)(xh.y - cen_y), hz = (float)(xh.z - cen_z);
            int2 my = cnt[hl];
            unsigned* row = nbr + (size_t)h * P.cap;
            const bool inside = FAST && fabsf(hx) <= P.hlx && fabsf(hy) <= P.hly && fabsf(hz) <= P.hlz;
            if (inside) {
#pragma unroll 4
                for (int k = 0; k < tn; k++) {
                    const float4 cp = cpos[k];
                    const float dx = hx - cp.x, dy = hy - cp.y, dz = hz - cp.z;
                    const float r2 = dx * dx + dy * dy + dz * dz;
                    if (r2 < P.r2hi) {
                        const unsigned tag = ctag[k];
                        const int j = (int)(tag & (P.skin ? kSkinIdxMask : 0x3fffffffu));
                        bool acc = r2 < P.r2lo;
                        if (!acc) acc = exact_r2(xh, xq[j], P.box) < P.rcut2;
                        if (acc && j != h && (!P.skin || half_keep(P, tag, j, h))) {
                            const unsigned dir = tag >> 30;
                            const unsigned isa = dir == 0 ? (unsigned)(h < j) : (unsigned)(dir == 1);
                            list_append(row, my, P.cap, P.skin ? tag : (unsigned)j | (isa << 31), __float_as_int(cp.w));
                        }
                    }
                }
            } else {
                for (int k = 0; k < tn; k++) {
                    const unsigned tag = ctag[k];
                    const int j = (int)(tag & (P.skin ? kSkinIdxMask : 0x3fffffffu));
                    if (j == h || (P.skin && !half_keep(P, tag, j, h))) continue;
                    if (exact_r2(xh, xq[j], P.box) < P.rcut2) {
                        const unsigned dir = tag >> 30;
                        const unsigned isa = dir == 0 ? (unsigned)(h < j) : (unsigned)(dir == 1);
                        list_append(row, my, P.cap, P.skin ? tag : (unsigned)j | (isa << 31),
                                    __float_as_int(cpos[k].w));
                    }
                }
            }
            cnt[hl] = my;
        }
    }
    __syncthreads();
    int lmax = 0;
    unsigned long long ltot = 0;
    for (int hl = tid; hl < nh; hl += blockDim.x) {
        const int2 m = cnt[hl];
        const int tot = m.x + m.y;
        if (tot > P.cap) {
            atomicOr(status, ST_NBR_OVERFLOW);
            nn[h0 + hl] = make_int2(0, 0);
        } else {
            nn[h0 + hl] = m;
        }
        lmax = max(lmax, tot);
        ltot += (unsigned long long)tot;
    }
    atomicMax(nn_max, lmax);
    atomicAdd(nn_tot, ltot);
}
template <bool FAST>
__global__ void __launch_bounds__(LB_THREADS)
    build_list_kernel(const int* __restrict__ cell_start, const int* __restrict__ entries,
                      const double4* __restrict__ xq, const int* __restrict__ ts, unsigned* __restrict__ nbr,
                      int2* __restrict__ nn, const __grid_constant__ LBParams P, int* __restrict__ status,
                      int* __restrict__ nn_max, unsigned long long* __restrict__ nn_tot,
                      const int* __restrict__ cond) {
    build_list_body<FAST>(own_blk(), cell_start, entries, xq, ts, nbr, nn, P, status, nn_max, nn_tot, cond);
}

int build_list(simox_ctx* c) {
    if (!c->gathered) {
        int st = gather_sorted(c);
        if (st) return st;
    }
    memset_async(c, c->nn_max, 0, sizeof(int), c->stream);
    memset_async(c, c->nn_tot, 0, sizeof(unsigned long long), c->stream);
    LBParams P;
    P.box = make_double3(c->box[0], c->box[1], c->box[2]);
    P.ibox = make_double3(c->inv_box[0], c->inv_box[1], c->inv_box[2]);
    P.origin = make_double3(-c->hbox[0], -c->hbox[1], -c->hbox[2]);
    P.skin = 0;
    P.half = 0;
    P.lc = make_double3(c->lc[0], c->lc[1], c->lc[2]);
    P.nc = make_int3(c->nc[0], c->nc[1], c->nc[2]);
    P.rcut2 = c->rcut2;
    P.r2lo = (float)(c->rcut2 * (1.0 - 4.0e-5));
    P.r2hi = (float)(c->rcut2 * (1.0 + 4.0e-5));
    P.hlx = (float)(0.5 * c->lc[0] + 1.0e-3);
    P.hly = (float)(0.5 * c->lc[1] + 1.0e-3);
    P.hlz = (float)(0.5 * c->lc[2] + 1.0e-3);
    P.cap = c->nnb_cap;
    P.npt_max = c->npt_max;
    size_t smem = LB_TILE * (sizeof(float4) + sizeof(unsigned)) + sizeof(int2) * c->npt_max;
    {
        Launch L(c, "neighbor_list");
        if (c->fast_cells)
            launch_k<LB_THREADS, 1, build_list_body<true>>(c, build_list_kernel<true>, c->ncell, smem, c->stream,
                c->cell_start, c->entries, c->xq_s, c->t_s, c->nbr, reinterpret_cast<int2*>(c->nn), P, c->status,
                c->nn_max, c->nn_tot, nullptr);
        else
            launch_k<LB_THREADS, 1, build_list_body<false>>(c, build_list_kernel<false>, c->ncell, smem, c->stream,
                c->cell_start, c->entries, c->xq_s, c->t_s, c->nbr, reinterpret_cast<int2*>(c->nn), P, c->status,
                c->nn_max, c->nn_tot, nullptr);
    }
    int st = check_launch(c);
    if (st) return st;
    c->list_valid = true;
    return SIMOX_OK;
}

// ---------------------------------------------------------------------------
// Verlet skin list.
//
// With fresh reference cells, at least 3 cells per axis and every atom inside
// [-L/2, L/2], the reference's pair set (atoms of adjacent cells with r2 <
// Rcut2) is exactly the set of minimum-image pairs with r2 < Rcut2.  The pair
// kernels then run in a private order (atoms binned on a grid of cells >=
// Rcut + skin) on a list filtered every step from a skin list (cutoff Rcut +
// skin).  The order and the skin list are rebuilt, on the device, when an atom
// has moved more than skin/2 since the last rebuild.  The filter (pair.cu,
// filter_density) applies the reference's exact FP64 r2 < Rcut2 test,
// recomputes from the current reference cells which atom of each pair is the
// reference's "i" (RDF), and accumulates the EAM densities of the kept pairs.

// rebuild flag: 1 if any atom moved more than skin/2 since the last rebuild
// (minimum image: an atom that VV_NVE1 wrapped across the box has not moved by L)
__device__ __forceinline__ void skin_check_body(Blk B, int n, const double* __restrict__ x,
                                                const double* __restrict__ x0, double3 box, double3 ibox, double lim2,
                                                int* __restrict__ flag) {
    const int i = B.x * blockDim.x + threadIdx.x;
    bool need = false;
    if (i < n) {
        double dx = x[3 * i] - x0[3 * i], dy = x[3 * i + 1] - x0[3 * i + 1], dz = x[3 * i + 2] - x0[3 * i + 2];
        dx -= box.x * rint(dx * ibox.x);
        dy -= box.y * rint(dy * ibox.y);
        dz -= box.z * rint(dz * ibox.z);
        need = !(dx * dx + dy * dy + dz * dz <= lim2);
    }
    if (__any_sync(0xffffffffu, need) && (threadIdx.x & 31) == 0) atomicOr(flag, 1);
}
__global__ void skin_check_kernel(int n, const double* __restrict__ x, const double* __restrict__ x0, double3 box,
                                  double3 ibox, double lim2, int* __restrict__ flag) {
    skin_check_body(own_blk(), n, x, x0, box, ibox, lim2, flag);
}

// bin on the skin grid and remember the positions of this rebuild;
// cond[0] = rebuild flag, cond[1] counts the rebuilds
__device__ __forceinline__ void skin_bin_body(Blk B, int n, const double* __restrict__ x, double3 hbox, double3 ilc,
                                              int3 nc, int* __restrict__ cell_of, int* __restrict__ count,
                                              double* __restrict__ x0, int* __restrict__ cond) {
    if (cond[0] == 0) return;
    const int i = B.x * blockDim.x + threadIdx.x;
    if (i == 0) cond[1] += 1;
    if (i >= n) return;
    const double xx[3] = {x[3 * i], x[3 * i + 1], x[3 * i + 2]};
    const double h[3] = {hbox.x, hbox.y, hbox.z}, il[3] = {ilc.x, ilc.y, ilc.z};
    const int m[3] = {nc.x, nc.y, nc.z};
    int id[3];
#pragma unroll
    for (int d = 0; d < 3; d++) {
        int v = (int)floor((xx[d] + h[d]) * il[d]);
        v = v < 0 ? 0 : (v >= m[d] ? m[d] - 1 : v);
        id[d] = v;
        x0[3 * i + d] = xx[d];
    }
    const int c = id[0] + id[1] * m[0] + id[2] * m[0] * m[1];
    cell_of[i] = c;
    atomicAdd(count + c, 1);
}
__global__ void skin_bin_kernel(int n, const double* __restrict__ x, double3 hbox, double3 ilc, int3 nc,
                                int* __restrict__ cell_of, int* __restrict__ count, double* __restrict__ x0,
                                int* __restrict__ cond) {
    skin_bin_body(own_blk(), n, x, hbox, ilc, nc, cell_of, count, x0, cond);
}

// Choose the pair-kernel order for the current state and gather into it.  In
// skin mode this also runs the (device-conditional) rebuild of the order and
// of the skin list.
static int prepare_order(simox_ctx* c) {
    const bool skin = c->skin_mode && c->cells_fresh && c->in_box;
    const int n = c->n;
    cudaStream_t s = c->stream;
    if (!skin) {
        if (int st = ensure_cell_lists(c)) return st;
        c->pair_order = c->sorted;
        c->using_skin = false;
        return gather_sorted(c);
    }
    c->pair_order = c->perm;
    c->using_skin = true;
    // the half list needs one metal species plus oxygen (the packed pair
    // kernels' tables); a new atom set invalidates the skin list, so the
    // choice holds for the list's whole life
    c->skin_half = c->precision != SIMOX_FP64 && c->g0_species >= 0;
    int* flag = c->skin_flag;
    if (!c->skin_valid) {
        // a new atom set: the first list is seeded from the host (not batched)
        if (c->rec) c->rec->bad = true;
        const int one = 1;
        cudaMemcpyAsync(flag, &one, sizeof(int), cudaMemcpyHostToDevice, s);
    } else {
        memset_async(c, flag, 0, sizeof(int), s);
        if (n > 0) {
            Launch L(c, "skin_check");
            const double h = 0.5 * c->skin;
            launch_k<256, 1, skin_check_body>(c, skin_check_kernel, (n + 255) / 256, 0, s, n, c->x, c->x0,
                make_double3(c->box[0], c->box[1], c->box[2]),
                make_double3(c->inv_box[0], c->inv_box[1], c->inv_box[2]), h * h, flag);
        }
    }
    // conditional rebuild of the order (binning on the skin grid)
    memset_async(c, c->cs_count, 0, sizeof(int) * c->ncell_s, s);
    if (n > 0) {
        Launch L(c, "skin_bin");
        launch_k<256, 1, skin_bin_body>(c, skin_bin_kernel, (n + 255) / 256, 0, s, n, c->x,
            make_double3(c->hbox[0], c->hbox[1], c->hbox[2]),
            make_double3(1.0 / c->lcs[0], 1.0 / c->lcs[1], 1.0 / c->lcs[2]),
            make_int3(c->ncs[0], c->ncs[1], c->ncs[2]), c->cs_cell_of, c->cs_count, c->x0, flag);
    }
    {
        Launch L(c, "skin_scan");
        launch_k<1024, 1, scan_cells_body>(c, scan_cells_kernel, 1, 0, s, c->cs_count, c->cs_start, c->cs_fill,
            c->ncell_s, c->npt_max_s, c->status, flag);
    }
    if (n > 0) {
        Launch L(c, "skin_scatter");
        launch_k<256, 1, scatter_atoms_body>(c, scatter_atoms_kernel, (n + 255) / 256, 0, s, n, c->cs_cell_of,
            c->cs_fill, c->perm, flag);
    }
    {
        Launch L(c, "skin_order");
        launch_k<128, 1, cell_rank_sort_body>(c, cell_rank_sort_kernel, c->ncell_s, sizeof(int) * c->npt_max_s, s,
            c->cs_start, c->perm, c->npt_max_s, flag);
    }
    int st = gather_sorted(c);
    if (st) return st;
    // conditional skin list build on the new order
    LBParams P;
    P.box = make_double3(c->box[0], c->box[1], c->box[2]);
    P.ibox = make_double3(c->inv_box[0], c->inv_box[1], c->inv_box[2]);
    P.origin = make_double3(-c->hbox[0], -c->hbox[1], -c->hbox[2]);
    P.lc = make_double3(c->lcs[0], c->lcs[1], c->lcs[2]);
    P.nc = make_int3(c->ncs[0], c->ncs[1], c->ncs[2]);
    const double rs = c->rcut + c->skin;
    P.rcut2 = rs * rs * (1.0 + 1.0e-4);
    P.r2lo = P.r2hi = (float)P.rcut2;   // a superset is enough: no exact test here
    P.hlx = (float)(0.5 * c->lcs[0] + 1.0e-3);
    P.hly = (float)(0.5 * c->lcs[1] + 1.0e-3);
    P.hlz = (float)(0.5 * c->lcs[2] + 1.0e-3);
    P.cap = c->cap_s;
    P.npt_max = c->npt_max_s;
    P.skin = 1;
    P.half = c->skin_half ? 1 : 0;
    const size_t smem = LB_TILE * (sizeof(float4) + sizeof(unsigned)) + sizeof(int2) * c->npt_max_s;
    {
        Launch L(c, "skin_list");
        launch_k<LB_THREADS, 1, build_list_body<true>>(c, build_list_kernel<true>, c->ncell_s, smem, s, c->cs_start,
            c->cs_entries, c->xq_s, c->t_s, c->nbr_s, reinterpret_cast<int2*>(c->nn_s), P, c->status, c->nn_max,
            c->nn_tot, flag);
    }
    c->skin_valid = true;
    return check_launch(c);
}

static int filter_list(simox_ctx* c) {
    memset_async(c, c->nn_max, 0, sizeof(int), c->stream);
    memset_async(c, c->nn_tot, 0, sizeof(unsigned long long), c->stream);
    int st = filter_density(c);
    if (st) return st;
    c->list_valid = true;
    return SIMOX_OK;
}

int ensure_gathered(simox_ctx* c) {
    if (!c->cells_valid) return SIMOX_E_STATE;
    if (c->gathered) return SIMOX_OK;
    c->list_valid = false;
    return prepare_order(c);
}

int ensure_list(simox_ctx* c) {
    int st = ensure_gathered(c);
    if (st) return st;
    if (c->list_valid) return SIMOX_OK;
    return c->using_skin ? filter_list(c) : build_list(c);
}

int setup_skin(simox_ctx* c) {
    c->skin_mode = false;
    if (!c->fast_cells || !(c->skin > 0.0)) return SIMOX_OK;
    const double rs = c->rcut + c->skin;
    // filter records: reference cells packed in 9 bits per axis, atom index
    // below the stencil code bits of a skin entry
    if ((size_t)c->cap > (size_t)kSkinIdxMask) return SIMOX_OK;
    for (int d = 0; d < 3; d++) {
        if (c->nc[d] > 511) return SIMOX_OK;
        c->ncs[d] = (int)(c->box[d] / rs);
        if (c->ncs[d] < 3) return SIMOX_OK;
        c->lcs[d] = c->box[d] / (double)c->ncs[d];
        if (!(0.5 * c->box[d] - rs - 0.5 * c->lcs[d] > 0.01)) return SIMOX_OK;
        // a listed pair stays closer than L/2 until the next rebuild
        if (!(0.5 * c->box[d] - 1.0001 * rs - c->skin > 0.01)) return SIMOX_OK;
    }
    c->ncell_s = c->ncs[0] * c->ncs[1] * c->ncs[2];
    const size_t N = (size_t)std::max(c->cap, 1);
    bool ok = cudaMalloc(&c->cs_count, sizeof(int) * c->ncell_s) == cudaSuccess &&
              cudaMalloc(&c->cs_start, sizeof(int) * (c->ncell_s + 1)) == cudaSuccess &&
              cudaMalloc(&c->cs_fill, sizeof(int) * c->ncell_s) == cudaSuccess &&
              cudaMalloc(&c->cs_cell_of, sizeof(int) * N) == cudaSuccess &&
              cudaMalloc(&c->cs_entries, sizeof(int) * c->ncell_s * kEntries) == cudaSuccess &&
              cudaMalloc(&c->perm, sizeof(int) * N) == cudaSuccess &&
              cudaMalloc(&c->x0, sizeof(double) * 3 * N) == cudaSuccess &&
              cudaMalloc(&c->skin_flag, 2 * sizeof(int)) == cudaSuccess &&
              cudaMemset(c->skin_flag, 0, 2 * sizeof(int)) == cudaSuccess &&
              cudaMalloc(&c->nn_s, sizeof(int) * 2 * N) == cudaSuccess &&
              cudaMalloc(&c->nbr_s, sizeof(unsigned) * N * (size_t)c->cap_s) == cudaSuccess;
    if (!ok) return SIMOX_E_NOMEM;
    // 27-cell stencil of the skin grid (distinct cells: >= 3 per axis)
    std::vector<int> E((size_t)c->ncell_s * kEntries);
    for (int k = 0; k < c->ncs[2]; k++)
        for (int j = 0; j < c->ncs[1]; j++)
            for (int i = 0; i < c->ncs[0]; i++) {
                const int cc = i + c->ncs[0] * (j + c->ncs[1] * k);
                int e = 0;
                for (int dk = -1; dk <= 1; dk++)
                    for (int dj = -1; dj <= 1; dj++)
                        for (int di = -1; di <= 1; di++) {
                            const int ii = (i + di + c->ncs[0]) % c->ncs[0];
                            const int jj = (j + dj + c->ncs[1]) % c->ncs[1];
                            const int kk = (k + dk + c->ncs[2]) % c->ncs[2];
                            E[(size_t)cc * kEntries + e++] = ii + c->ncs[0] * (jj + c->ncs[1] * kk);
                        }
            }
    if (cudaMemcpyAsync(c->cs_entries, E.data(), E.size() * sizeof(int), cudaMemcpyHostToDevice, c->stream) !=
        cudaSuccess)
        return SIMOX_E_CUDA;
    c->skin_mode = true;
    c->skin_valid = false;
    return cuda_status(cudaStreamSynchronize(c->stream));
}

int list_prepare(simox_ctx* c) {
    // a permission, not a reservation: each launch passes its own size
    const int bytes = std::max(96 * 1024, (int)(LB_TILE * (sizeof(float4) + sizeof(unsigned)) +
                                                sizeof(int2) * std::max(c->npt_max, c->npt_max_s)));
    cudaError_t e1 = cudaFuncSetAttribute(build_list_kernel<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
    cudaError_t e2 = cudaFuncSetAttribute(build_list_kernel<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
    if (e1 != cudaSuccess || e2 != cudaSuccess) return SIMOX_E_ARG;
    return SIMOX_OK;
}

}  // namespace sx
