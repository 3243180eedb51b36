// pair_half.cu -- the mixed-precision pair passes on a half neighbour list.
//
// In skin mode with one metal species plus oxygen, a mixed-precision context
// keeps every pair once: the skin row of atom X holds the partners Y in the 13
// forward cells of X's skin cell (stencil positions 14..26) and those in X's
// own cell with a later pair-order index (position 13).  Each pair's terms
// are evaluated once.  X's share stays in registers; Y's share is added into
// accumulators in shared memory that cover the 14 cells one CTA can reach (its
// "tile"), and each CTA adds its tile into the global accumulators once.
//
// Every accumulator is a 64-bit fixed-point integer: a term v is added as
// round(v * 2^s).  Integer addition is associative, so the sums -- densities,
// forces, the charge solver's matrix-vector products -- do not depend on the
// order in which warps and CTAs add them, and every run gives the same bits.
// Scales: densities and charge-solver sums 2^40 (range 8.4e6, resolution
// 9.1e-13), forces 2^32 (range 2.1e9 eV/A, resolution 2.3e-10 eV/A).
//
//   pass 1 (filter_half_kernel): the skin filter (the reference's FP64
//          r2 < Rcut2 test near the cutoff, force.f90:51-54) and both
//          densities of each kept pair (force.f90:84-85); kept entries are
//          compacted into the exact half row.  embed_half_kernel then forms
//          F'(rho) (force.f90:256-351).
//   pass 2 (force_half_kernel): the pair force of force.f90:81-98 and
//          101-140 with the density back-pass of force.f90:353-358 folded in,
//          once per pair, on packed FP32 (two entries per lane), and the RDF
//          (force.f90:76,180), each pair counted once under the reference's
//          (i, j) species order; on RDF steps the pass finds which atom of a
//          pair is the reference's i from the reference cells
//          (cellsort.f90:18-30), so ordinary steps skip that work.
//   charge solver (ctip_half_kernel): sum_Y sym_XY v_Y and chi + sum_Y
//          Z_Y asym_XY of ctip.f90:85-110 and dUdq (ctip.f90:307-333).
//   energies (energy_half_kernel): the FP64 pair energies once per pair and
//          the FP64 densities for the embedding energy.
#include "simox_pair.cuh"

#include <atomic>

namespace sx {

typedef unsigned long long u64;

constexpr float kRhoScale = 1099511627776.0f;            // 2^40
constexpr double kRhoScaleD = 1099511627776.0;
constexpr double kRhoUnit = 1.0 / 1099511627776.0;
constexpr float kForceScale = 4294967296.0f;              // 2^32
constexpr double kForceScaleD = 4294967296.0;
constexpr double kForceUnit = 1.0 / 4294967296.0;
constexpr float kForceMax = 1.0e9f;                       // |term| beyond this: out of range
constexpr int kHalfFirst = 13;                            // stencil position of the own cell
constexpr int kHalfCells = 14;                            // positions 13..26
constexpr int kSelf = 13;

// pass 1: 256 threads, shared density accumulators for up to 4,096 tile atoms
constexpr int kH1Threads = 256;
constexpr int kH1Cap = 4096;
// pass 2 and the charge solver: 1024 threads (64 registers), one CTA per SM,
// dynamic tiles; 32 resident warps hide the pair function's latency chains
// (0.407 ms for the 128k corundum force pass against 0.43 ms at 512 threads)
constexpr int kH2Threads = 1024;
constexpr int kH2Cap = 3584;                              // 60 B per atom: 210 KB
constexpr size_t kH2Smem = (size_t)kH2Cap * (sizeof(double4) + sizeof(float) + 6 * sizeof(unsigned));
constexpr int kHCCap = 4608;                              // 40 B per atom: 184 KB
constexpr size_t kHCSmem = (size_t)kHCCap * (sizeof(float4) + sizeof(double) + 4 * sizeof(unsigned));

__device__ __forceinline__ void add_fixed(u64* p, long long v) { atomicAdd(p, (u64)v); }

// The 14 cells of a CTA's tile: first pair-order index of each and their
// offsets in the tile (own cell first).
struct HalfTile {
    int start[kHalfCells];
    int off[kHalfCells + 1];
};

// A 64-bit fixed-point sum in shared memory held as two 32-bit words: the
// carry out of the low word goes into the high word, so the pair adds up
// exactly (modulo 2^64) in any order.  Two 32-bit shared atomics run several
// times faster than one 64-bit shared atomic on this GPU, and measured
// faster in the pair passes than independent low/high parts added without
// the carry (whose range check costs more than the returned value's wait).
__device__ __forceinline__ void add_split(unsigned* lo, unsigned* hi, int i, long long v) {
    const unsigned vl = (unsigned)v, vh = (unsigned)((unsigned long long)v >> 32);
    const unsigned old = atomicAdd(lo + i, vl);
    atomicAdd(hi + i, vh + ((unsigned)(old + vl) < old ? 1u : 0u));
}

__device__ __forceinline__ long long slot_value(unsigned lo, unsigned hi) {
    return (long long)(((unsigned long long)hi << 32) | lo);
}

// Where a partner's share goes: the CTA's tile (split words, `stride` slots
// per component) or, for a tile too large for shared memory, the global
// 64-bit sums (`stride` entries per component, pair order).  X's own row sum
// goes to the global sum in both cases.
template <bool TILED> struct Sink;
template <> struct Sink<true> {
    unsigned* lo;
    unsigned* hi;
    int stride;
    u64* g;
    int gstride;
    __device__ __forceinline__ void add(int c, int i, long long v) const { add_split(lo + c * stride, hi + c * stride, i, v); }
    __device__ __forceinline__ void own(int c, int X, long long v) const {
        atomicAdd(g + (size_t)c * gstride + X, (u64)v);
    }
};
template <> struct Sink<false> {
    u64* g;
    int stride;
    __device__ __forceinline__ void add(int c, int i, long long v) const { atomicAdd(g + (size_t)c * stride + i, (u64)v); }
    __device__ __forceinline__ void own(int c, int X, long long v) const { add(c, X, v); }
};

__device__ __forceinline__ void half_tile_setup(HalfTile& T, const int* __restrict__ cs_start,
                                                const int* __restrict__ cs_entries, int cell) {
    const int tid = threadIdx.x;
    if (tid < kHalfCells) {
        const int nc = cs_entries[cell * kEntries + kHalfFirst + tid];
        const int s0 = cs_start[nc];
        T.start[tid] = s0;
        T.off[tid + 1] = cs_start[nc + 1] - s0;
    }
    if (tid == 0) T.off[0] = 0;
    __syncthreads();
    if (tid == 0)
        for (int t = 0; t < kHalfCells; t++) T.off[t + 1] += T.off[t];
    __syncthreads();
}

// X range [b0, b1) of CTA part `part` of `splits` over the own cell
__device__ __forceinline__ int2 half_range(const HalfTile& T, int part, int splits) {
    const int a0 = T.start[0], na = T.off[1];
    return make_int2(a0 + (int)((long long)na * part / splits), a0 + (int)((long long)na * (part + 1) / splits));
}

// Adds the tile's sums (nacc components of `stride` slots) into the global
// 64-bit sums (nacc components of `gstride`), skipping zeros.
__device__ __forceinline__ void half_tile_flush(const HalfTile& T, int total, const unsigned* lo,
                                                const unsigned* hi, int stride, int nacc, u64* gacc, int gstride) {
    int t = 0;
    for (int i = threadIdx.x; i < total; i += blockDim.x) {
        while (T.off[t + 1] <= i) t++;
        const int gi = T.start[t] + (i - T.off[t]);
        for (int a = 0; a < nacc; a++) {
            const long long v = slot_value(lo[a * stride + i], hi[a * stride + i]);
            if (v) atomicAdd(gacc + (size_t)a * gstride + gi, (u64)v);
        }
    }
}

// ---------------------------------------------------------------------------
// pass 1

struct Half1Params {
    FilterParams F;
    int splits, g0;
};

// One group of X's half skin row (G = 0: metal partners of species g0 at the
// row front; G = 1: oxygen at the back).  Kept entries are compacted into X's
// exact half row; their density at X
// is summed in rho and their density at Y is added to Y's accumulator.
template <int G, bool TILED>
__device__ __forceinline__ int filter_group_half(const Half1Params& H, const float4* ssh, const DensC<float>& du,
                                                 const DensC<float>& dv, int sX, int sY,
                                                 const unsigned* __restrict__ sp, int mg, unsigned* __restrict__ dp,
                                                 const float4& ra, int X, const double4* __restrict__ xq,
                                                 const float4* __restrict__ rec, const int* delta, int lim,
                                                 const Sink<TILED>& acc, double& rho) {
    const FilterParams& F = H.F;
    const PairParams& P = F.pp;
    const int lane = threadIdx.x & 31;
    const unsigned lt = (1u << lane) - 1u;
    auto ent = [&](int k) { return k < mg ? sp[G == 0 ? k : -k] : 0u; };
    unsigned E1 = ent(lane), E2 = ent(lane + 32);
    float4 rb1 = rec[E1 & kSkinIdxMask];
    int out = 0;
    for (int base = 0; base < mg; base += 32) {
        const int k = base + lane;
        const unsigned e = E1;
        const float4 rb = rb1;
        E1 = E2;
        rb1 = rec[E1 & kSkinIdxMask];
        E2 = ent(k + 64);
        const unsigned Y = e & kSkinIdxMask;
        const int code = (int)(e >> kSkinCodeShift);
        const bool live = k < mg;
        const float4 o = ssh[code];
        const float dx = (rb.x - ra.x) + o.x, dy = (rb.y - ra.y) + o.y, dz = (rb.z - ra.z) + o.z;
        const float r2 = fmaf(dx, dx, fmaf(dy, dy, dz * dz));
        bool keep = live & (r2 < F.rcut2f);
        const bool inband = live & (fabsf(r2 - F.rcut2f) <= F.band);
        if (__any_sync(0xffffffffu, inband)) {
            if (inband) {   // within FP32 rounding of the cutoff: the reference's FP64 test
                double ddx, ddy, ddz;
                min_image(xq[X], xq[Y], P, ddx, ddy, ddz);
                keep = __dadd_rn(__dadd_rn(__dmul_rn(ddx, ddx), __dmul_rn(ddy, ddy)), __dmul_rn(ddz, ddz)) < F.rcut2;
            }
        }
        const unsigned mask = __ballot_sync(0xffffffffu, keep);
        const int pos = out + __popc(mask & lt);
        if (keep & (pos < P.cap)) dp[G == 0 ? pos : -pos] = e;
        out += __popc(mask);
        const float r = r2 * rsqrt_approx(r2);
        // a same-species pair contributes the same density to both atoms
        // (sX == sY is uniform across the warp: one X, one partner group)
        const float vX = dens_term<float>(du, r), vY = sX == sY ? vX : dens_term<float>(dv, r);
        rho += keep ? (double)vX : 0.0;
        if (keep) {
            // stencil positions below 13 never occur in a half row: clamp into range anyway
            int slot = TILED ? (int)Y + delta[max(code - kHalfFirst, 0)] : (int)Y;
            slot = (unsigned)slot < (unsigned)lim ? slot : 0;
            acc.add(0, slot, __float2ll_rn(vY * kRhoScale));
        }
    }
    return out;
}

template <bool TILED>
__device__ __forceinline__ void filter_half_atoms(const Half1Params& H, const float4* ssh, const DensC<float>* dsh,
                                                  int b0, int b1, int a0, int* next, const double4* __restrict__ xq,
                                                  const float4* __restrict__ rec, const int* __restrict__ order,
                                                  const int2* __restrict__ nn_s, const unsigned* __restrict__ nbr_s,
                                                  int2* __restrict__ nn, unsigned* __restrict__ nbr, const int* delta,
                                                  int lim, const Sink<TILED>& acc, int& lmax, unsigned long long& ltot,
                                                  int& bad) {
    const FilterParams& F = H.F;
    const int lane = threadIdx.x & 31;
    const int g0 = H.g0;
    for (;;) {
        int X = 0;
        if (lane == 0) X = atomicAdd(next, 1);
        X = __shfl_sync(0xffffffffu, X, 0) + b0;
        if (X >= b1) break;
        const float4 ra = rec[X];
        const unsigned wa = __float_as_uint(ra.w);
        const int sX = (int)(wa >> 27);
        if (sX != g0 && sX != 3) {   // not on this path (cannot happen: checked by the host)
            bad |= ST_UNKNOWN_PAIR;
            if (lane == 0) nn[X] = make_int2(0, 0);
            continue;
        }
        const int2 ms = nn_s[X];
        const unsigned* srow = nbr_s + (size_t)X * F.cap_s;
        unsigned* row = nbr + (size_t)X * F.pp.cap;
        double rho = 0.0;
        const int out0 = filter_group_half<0, TILED>(H, ssh, dsh[(sX << 3) | g0], dsh[(g0 << 3) | sX], sX, g0,
                                                     srow, ms.x, row, ra, X, xq, rec, delta, lim, acc, rho);
        const int out1 = filter_group_half<1, TILED>(H, ssh, dsh[(sX << 3) | 3], dsh[(3 << 3) | sX], sX, 3,
                                                     srow + (F.cap_s - 1), ms.y, row + (F.pp.cap - 1), ra, X, xq,
                                                     rec, delta, lim, acc, rho);
        rho = warp_sum(rho);
        if (lane == 0) {
            const int tot = out0 + out1;
            if (tot > F.pp.cap) {
                bad |= ST_NBR_OVERFLOW;
                nn[X] = make_int2(0, 0);
            } else {
                nn[X] = make_int2(out0, out1);
            }
            lmax = max(lmax, tot);
            ltot += (unsigned long long)tot;
            acc.own(0, X, __double2ll_rn(rho * kRhoScaleD));
        }
    }
}

__device__ __forceinline__ void filter_half_body(Blk B, const Half1Params& H, const PairTab<float>* __restrict__ tab,
                                                 const double4* __restrict__ xq, const float4* __restrict__ rec,
                                                 const int* __restrict__ order, const int* __restrict__ cs_start,
                                                 const int* __restrict__ cs_entries, const int2* __restrict__ nn_s,
                                                 const unsigned* __restrict__ nbr_s, int2* __restrict__ nn,
                                                 unsigned* __restrict__ nbr, u64* __restrict__ rho_fx,
                                                 int* __restrict__ status, int* __restrict__ nn_max,
                                                 unsigned long long* __restrict__ nn_tot) {
    __shared__ unsigned alo[kH1Cap], ahi[kH1Cap];
    __shared__ DensC<float> dsh[64];
    __shared__ int dflag[64];
    __shared__ float4 ssh[kEntries];
    __shared__ HalfTile T;
    __shared__ int delta[kHalfCells];
    __shared__ int next;
    const int tid = threadIdx.x;
    for (int k = tid; k < 64; k += blockDim.x) {
        const int a = k >> 3, b = k & 7;
        DensC<float> d{};
        int fl = ST_UNKNOWN_PAIR;
        d.ire = 1.f;
        if (a < kSpecies && b < kSpecies) {
            const PairTab<float>& t = tab[a * kSpecies + b];
            d.fe = t.d_fe; d.ire = t.d_inv_re; d.c = t.d_c; d.lam = t.d_lam; d.nlam = -t.d_lam;
            d.k1 = -1.4426950408889634f * t.d_c * t.d_inv_re;
            d.k0 = 1.4426950408889634f * t.d_c;
            fl = t.valid ? 0 : ST_UNSUPPORTED;
        }
        dsh[k] = d;
        dflag[k] = fl;
    }
    for (int k = tid; k < kEntries; k += blockDim.x) ssh[k] = H.F.sh[k];
    if (tid == 0) next = 0;
    const int cell = B.x / H.splits, part = B.x - cell * H.splits;
    half_tile_setup(T, cs_start, cs_entries, cell);
    const int total = T.off[kHalfCells];
    const int2 br = half_range(T, part, H.splits);
    const int b0 = br.x, b1 = br.y;
    const bool tiled = total <= kH1Cap;
    if (tid < kHalfCells) delta[tid] = T.off[tid] - T.start[tid];
    if (tiled)
        for (int i = tid; i < total; i += blockDim.x) {
            alo[i] = 0u;
            ahi[i] = 0u;
        }
    __syncthreads();
    const int g0 = H.g0;
    const int a0 = T.start[0];
    int lmax = 0, bad = 0;
    unsigned long long ltot = 0;
    if (b1 > b0) {
        // the four pair kinds of this path (the metal g0 and oxygen)
        bad = dflag[(g0 << 3) | g0] | dflag[(g0 << 3) | 3] | dflag[(3 << 3) | g0] | dflag[(3 << 3) | 3];
        if (tiled)
            filter_half_atoms<true>(H, ssh, dsh, b0, b1, a0, &next, xq, rec, order, nn_s, nbr_s, nn, nbr, delta,
                                    total, Sink<true>{alo, ahi, 0, rho_fx, 0}, lmax, ltot, bad);
        else
            filter_half_atoms<false>(H, ssh, dsh, b0, b1, a0, &next, xq, rec, order, nn_s, nbr_s, nn, nbr, delta,
                                     H.F.pp.n, Sink<false>{rho_fx, 0}, lmax, ltot, bad);
    }
    if (bad) atomicOr(status, bad);
    if ((tid & 31) == 0) {
        if (lmax) atomicMax(nn_max, lmax);
        if (ltot) atomicAdd(nn_tot, ltot);
    }
    __syncthreads();
    if (tiled) half_tile_flush(T, total, alo, ahi, 0, 1, rho_fx, 0);
}
__global__ void __launch_bounds__(kH1Threads)
    filter_half_kernel(const __grid_constant__ Half1Params H, const PairTab<float>* __restrict__ tab,
                       const double4* __restrict__ xq, const float4* __restrict__ rec, const int* __restrict__ order,
                       const int* __restrict__ cs_start, const int* __restrict__ cs_entries,
                       const int2* __restrict__ nn_s, const unsigned* __restrict__ nbr_s, int2* __restrict__ nn,
                       unsigned* __restrict__ nbr, u64* __restrict__ rho_fx, int* __restrict__ status,
                       int* __restrict__ nn_max, unsigned long long* __restrict__ nn_tot) {
    filter_half_body(own_blk(), H, tab, xq, rec, order, cs_start, cs_entries, nn_s, nbr_s, nn, nbr, rho_fx, status,
        nn_max, nn_tot);
}

// rho from the fixed-point sums, then F'(rho) (force.f90:256-351)
__device__ __forceinline__ void embed_half_body(Blk B, int n, const int* __restrict__ ts,
                                                const u64* __restrict__ rho_fx, const EmbedParams& E,
                                                double* __restrict__ rho_s, double* __restrict__ dF_s,
                                                float* __restrict__ dF_f, int* __restrict__ status) {
    const int k = B.x * blockDim.x + threadIdx.x;
    if (k >= n) return;
    const double rho = (double)(long long)rho_fx[k] * kRhoUnit;
    double F, dF;
    if (embed(E, ts[k], rho, F, dF)) atomicOr(status, ST_UNKNOWN_ELEMENT);
    rho_s[k] = rho;
    dF_s[k] = dF;
    dF_f[k] = (float)dF;
}
__global__ void embed_half_kernel(int n, const int* __restrict__ ts, const u64* __restrict__ rho_fx,
                                  const __grid_constant__ EmbedParams E, double* __restrict__ rho_s,
                                  double* __restrict__ dF_s, float* __restrict__ dF_f, int* __restrict__ status) {
    embed_half_body(own_blk(), n, ts, rho_fx, E, rho_s, dF_s, dF_f, status);
}

// ---------------------------------------------------------------------------
// pass 2
//
// Separations are formed in FP64 and then rounded to FP32: each atom's record
// holds its FP64 offset from the centre of the skin cell it was binned into;
// the tile stores the partner cells' offsets already moved by their stencil
// shift o * Lcs, so x_X - x_Y = off_X - tile_Y exactly up to FP64 rounding.
// (Differences of FP32 offsets lose up to ~1e-6 A in the subtraction itself,
// which the stiff near-neighbour forces turn into per-atom errors near the
// 1e-5 bar.)

struct Half2Params {
    PackParams Q;
    double3 lcs;               // skin-cell edges
    int3 nc;                   // reference cell grid (RDF: the reference's i)
    int splits, g0, n, fstride;
};

// X's reference cell for the reference's-i test of the RDF: wa = X's record
// word (reference cell 9 bits per axis), the cells below X's on each axis
// (periodic) and X's reference order
struct RefX {
    unsigned wa;
    int xm, ym, zm, oX;
};

__device__ __forceinline__ RefX ref_x(const Half2Params& H, const float4* __restrict__ rec,
                                      const int* __restrict__ order, int X) {
    RefX R;
    R.wa = __float_as_uint(rec[X].w);
    const int ax = R.wa & 511, ay = (R.wa >> 9) & 511, az = (R.wa >> 18) & 511;
    R.xm = ax == 0 ? H.nc.x - 1 : ax - 1;
    R.ym = ay == 0 ? H.nc.y - 1 : ay - 1;
    R.zm = az == 0 ? H.nc.z - 1 : az - 1;
    R.oX = order[X];
    return R;
}

// X is the reference's i of the listed pair (X, Y): Y's reference cell is one
// of the 13 forward cells of X's (cellsort.f90:18-30), or the same cell and X
// comes first in the reference's order
__device__ __forceinline__ bool ref_isa(const RefX& R, const float4* __restrict__ rec,
                                        const int* __restrict__ order, int Y) {
    const unsigned wb = __float_as_uint(rec[Y].w);
    const int bx = wb & 511, by = (wb >> 9) & 511, bz = (wb >> 18) & 511;
    const int ay = (R.wa >> 9) & 511, az = (R.wa >> 18) & 511;
    const bool same = ((wb ^ R.wa) & 0x07ffffffu) == 0u;
    return (bz == R.zm) | ((bz == az) & ((by == R.ym) | ((by == ay) & ((bx == R.xm) | (same && R.oX < order[Y])))));
}

// o_e * Lcs of stencil position e = (dk+1) 9 + (dj+1) 3 + (di+1)
__device__ __forceinline__ double3 stencil_shift(int e, double3 lcs) {
    return make_double3((e % 3 - 1) * lcs.x, ((e / 3) % 3 - 1) * lcs.y, (e / 9 - 1) * lcs.z);
}

// Two entries of X's half row as the halves of packed FP32 values: f/r of
// each pair, X's share into the compensated FP32 sums, Y's share (the
// opposite force) into Y's fixed-point sums.
template <bool SAME, bool MHOMO, bool RDF, bool TILED, int TI>
__device__ __forceinline__ void force_half_batch(const Half2Params& H, const int* edelta, const double3* esh,
                                                 const double4* __restrict__ psrc, const float* __restrict__ dsrc,
                                                 int lim, unsigned E1, unsigned E2, bool v1, bool v2ok,
                                                 const double4& ra, float dFX, const Sink<TILED>& acc, v2 (&fh)[3],
                                                 v2 (&fl)[3], int* hist, const RefX& RX, const float4* __restrict__ rec,
                                                 const int* __restrict__ order, int& bad) {
    constexpr int NB = SIMOX_NRDF + 2;
    const PackParams& Q = H.Q;
    const PackTab& T = Q.tab[TI];
    const float qa = (float)ra.w;
    const float kcqa = Q.kc * qa;
    const float kcqaZY = T.kcZY * qa;
    const int c1 = min((int)((E1 >> kSkinCodeShift) & kCodeMask), kEntries - 1);
    const int c2 = min((int)((E2 >> kSkinCodeShift) & kCodeMask), kEntries - 1);
    int i1 = (int)(E1 & kIdxMask) + edelta[c1];
    int i2 = (int)(E2 & kIdxMask) + edelta[c2];
    // keep every access inside the tile (or the atom range)
    i1 = (unsigned)i1 < (unsigned)lim ? i1 : 0;
    i2 = (unsigned)i2 < (unsigned)lim ? i2 : 0;
    double4 P1 = psrc[i1], P2 = psrc[i2];
    if (!TILED) {   // global offsets: add the stencil shift here
        const double3 s1 = esh[c1], s2 = esh[c2];
        P1.x += s1.x; P1.y += s1.y; P1.z += s1.z;
        P2.x += s2.x; P2.y += s2.y; P2.z += s2.z;
    }
    const float D1 = dsrc[i1], D2 = dsrc[i2];
    const v2 dx = mk2((float)(ra.x - P1.x), (float)(ra.x - P2.x));
    const v2 dy = mk2((float)(ra.y - P1.y), (float)(ra.y - P2.y));
    const v2 dz = mk2((float)(ra.z - P1.z), (float)(ra.z - P2.z));
    const v2 r2 = fma2(dx, dx, fma2(dy, dy, dz * dz));
    v2 fs = pair_fs_pk<SAME, MHOMO>(T, Q, r2, mk2((float)P1.w, (float)P2.w), mk2(D1, D2), dFX, kcqa, kcqaZY);
    fs = mk2(v1 ? fs.v.x : 0.f, v2ok ? fs.v.y : 0.f);   // slots past the end of a group: placeholders
    const v2 px = fs * dx, py = fs * dy, pz = fs * dz;
    two_sum2(fh[0], fl[0], px);
    two_sum2(fh[1], fl[1], py);
    two_sum2(fh[2], fl[2], pz);
    if (v1) {
        if (!(fabsf(px.v.x) < kForceMax && fabsf(py.v.x) < kForceMax && fabsf(pz.v.x) < kForceMax)) bad |= ST_POSITION;
        acc.add(0, i1, -__float2ll_rn(px.v.x * kForceScale));
        acc.add(1, i1, -__float2ll_rn(py.v.x * kForceScale));
        acc.add(2, i1, -__float2ll_rn(pz.v.x * kForceScale));
    }
    if (v2ok) {
        if (!(fabsf(px.v.y) < kForceMax && fabsf(py.v.y) < kForceMax && fabsf(pz.v.y) < kForceMax)) bad |= ST_POSITION;
        acc.add(0, i2, -__float2ll_rn(px.v.y * kForceScale));
        acc.add(1, i2, -__float2ll_rn(py.v.y * kForceScale));
        acc.add(2, i2, -__float2ll_rn(pz.v.y * kForceScale));
    }
    if (RDF) {
        // INT(r/dr) of the pair's FP32 distance, once per pair, under the
        // species order of the reference's (i, j): TI is (X kind) * 2 + (Y kind)
        constexpr int kxy = TI, kyx = ((TI & 1) << 1) | (TI >> 1);
        if (v1) {
            const float r = r2.v.x * rsqrt_approx(r2.v.x);
            const bool isa = ref_isa(RX, rec, order, (int)(E1 & kIdxMask));
            atomicAdd(&hist[(isa ? kxy : kyx) * NB + min(max((int)(r * Q.inv_dr), 0), NB - 1)], 2);
        }
        if (v2ok) {
            const float r = r2.v.y * rsqrt_approx(r2.v.y);
            const bool isa = ref_isa(RX, rec, order, (int)(E2 & kIdxMask));
            atomicAdd(&hist[(isa ? kxy : kyx) * NB + min(max((int)(r * Q.inv_dr), 0), NB - 1)], 2);
        }
    }
}

template <bool TILED, bool RDF>
__device__ __forceinline__ void force_half_atoms(const Half2Params& H, const int* edelta, const double3* esh,
                                                 const double4* __restrict__ psrc, const float* __restrict__ dsrc,
                                                 int lim, int b0, int b1, int a0, int* next,
                                                 const double4* __restrict__ xo, const int* __restrict__ ts,
                                                 const int2* __restrict__ nn, const unsigned* __restrict__ nbr,
                                                 const float* __restrict__ dF_f, const Sink<TILED>& acc, int* hist,
                                                 const float4* __restrict__ rec, const int* __restrict__ order,
                                                 int& bad) {
    const int lane = threadIdx.x & 31;
    const int cap = H.Q.cap;
    const int g0 = H.g0;
    for (;;) {
        int X = 0;
        if (lane == 0) X = atomicAdd(next, 1);
        X = __shfl_sync(0xffffffffu, X, 0) + b0;
        if (X >= b1) break;
        const double4 ra = xo[X];
        const int sX = ts[X];
        const float dFX = dF_f[X];
        const RefX RX = RDF ? ref_x(H, rec, order, X) : RefX{};
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
            const unsigned pad = ((unsigned)kSelf << kSkinCodeShift) | (unsigned)X;   // an in-tile placeholder
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
                if (metal) {
                    if (!g1) force_half_batch<true, true, RDF, TILED, 0>(H, edelta, esh, psrc, dsrc, lim, E1, E2, v1, v2ok, ra, dFX, acc, fh, fl, hist, RX, rec, order, bad);
                    else force_half_batch<false, false, RDF, TILED, 1>(H, edelta, esh, psrc, dsrc, lim, E1, E2, v1, v2ok, ra, dFX, acc, fh, fl, hist, RX, rec, order, bad);
                } else {
                    if (!g1) force_half_batch<false, false, RDF, TILED, 2>(H, edelta, esh, psrc, dsrc, lim, E1, E2, v1, v2ok, ra, dFX, acc, fh, fl, hist, RX, rec, order, bad);
                    else force_half_batch<true, false, RDF, TILED, 3>(H, edelta, esh, psrc, dsrc, lim, E1, E2, v1, v2ok, ra, dFX, acc, fh, fl, hist, RX, rec, order, bad);
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
            acc.own(0, X, __double2ll_rn(fx * kForceScaleD));
            acc.own(1, X, __double2ll_rn(fy * kForceScaleD));
            acc.own(2, X, __double2ll_rn(fz * kForceScaleD));
        }
    }
}

template <bool RDF>
__device__ __forceinline__ void force_half_body(Blk B, const Half2Params& H, const int* __restrict__ cs_start,
                                                const int* __restrict__ cs_entries, const double4* __restrict__ xo,
                                                const int* __restrict__ ts, const int2* __restrict__ nn,
                                                const unsigned* __restrict__ nbr, const float* __restrict__ dF_f,
                                                u64* __restrict__ f_fx, int* __restrict__ rdf,
                                                const float4* __restrict__ rec, const int* __restrict__ order,
                                                int* __restrict__ status) {
    constexpr int NB = SIMOX_NRDF + 2;
    extern __shared__ __align__(16) unsigned char half_smem[];
    double4* tpos = reinterpret_cast<double4*>(half_smem);                 // partner offsets + shift, charge
    unsigned* tlo = reinterpret_cast<unsigned*>(tpos + kH2Cap);            // [3][cap] low words
    unsigned* thi = tlo + 3 * kH2Cap;                                      // [3][cap] high words
    float* tdf = reinterpret_cast<float*>(thi + 3 * kH2Cap);               // F'
    __shared__ double3 esh[kEntries];          // o_e * Lcs
    __shared__ int edelta[kEntries];           // tile index delta of each stencil position
    __shared__ HalfTile T;
    __shared__ int next;
    __shared__ int hist[RDF ? 4 * NB : 1];     // (metal, O) x (metal, O) kinds of the reference's (i, j)
    const int tid = threadIdx.x;
    const int cell = B.x / H.splits, part = B.x - cell * H.splits;
    if (tid == 0) next = 0;
    if (RDF)
        for (int k = tid; k < 4 * NB; k += kH2Threads) hist[k] = 0;
    half_tile_setup(T, cs_start, cs_entries, cell);
    const int total = T.off[kHalfCells];
    const int2 br = half_range(T, part, H.splits);
    const int b0 = br.x, b1 = br.y;
    const bool tiled = total <= kH2Cap;
    if (tid < kEntries) {
        esh[tid] = stencil_shift(tid, H.lcs);
        // positions below 13 never occur in a half row: a delta that the
        // range clamp maps to slot 0
        edelta[tid] = tid < kHalfFirst ? -(1 << 28) : (tiled ? T.off[tid - kHalfFirst] - T.start[tid - kHalfFirst] : 0);
    }
    __syncthreads();
    if (tiled) {
        int t = 0;
        for (int i = tid; i < total; i += kH2Threads) {
            while (T.off[t + 1] <= i) t++;
            const int src = T.start[t] + (i - T.off[t]);
            const double3 sh = esh[kHalfFirst + t];
            double4 p = xo[src];
            p.x += sh.x;
            p.y += sh.y;
            p.z += sh.z;
            tpos[i] = p;
            tdf[i] = dF_f[src];
#pragma unroll
            for (int c = 0; c < 3; c++) {
                tlo[c * kH2Cap + i] = 0u;
                thi[c * kH2Cap + i] = 0u;
            }
        }
    }
    __syncthreads();
    const int a0 = T.start[0];
    int bad = 0;
    if (tiled)
        force_half_atoms<true, RDF>(H, edelta, esh, tpos, tdf, total, b0, b1, a0, &next, xo, ts, nn, nbr, dF_f,
                                    Sink<true>{tlo, thi, kH2Cap, f_fx, H.fstride}, hist, rec, order, bad);
    else
        force_half_atoms<false, RDF>(H, edelta, esh, xo, dF_f, H.n, b0, b1, a0, &next, xo, ts, nn, nbr, dF_f,
                                     Sink<false>{f_fx, H.fstride}, hist, rec, order, bad);
    if (bad) atomicOr(status, bad);
    __syncthreads();
    if (tiled) half_tile_flush(T, total, tlo, thi, kH2Cap, 3, f_fx, H.fstride);
    if (RDF) {
        const int g0 = H.g0;
        for (int k = tid; k < 4 * NB; k += kH2Threads) {
            const int v = hist[k];
            if (v) {
                const int kind = k / NB, bin = k - kind * NB;
                const int si = (kind >> 1) ? 3 : g0, sj = (kind & 1) ? 3 : g0;
                atomicAdd(&rdf[si + 5 * sj + 25 * bin], v);
            }
        }
    }
}
template <bool RDF>
__global__ void __launch_bounds__(kH2Threads, 1)
    force_half_kernel(const __grid_constant__ Half2Params H, const int* __restrict__ cs_start,
                      const int* __restrict__ cs_entries, const double4* __restrict__ xo, const int* __restrict__ ts,
                      const int2* __restrict__ nn, const unsigned* __restrict__ nbr, const float* __restrict__ dF_f,
                      u64* __restrict__ f_fx, int* __restrict__ rdf, const float4* __restrict__ rec,
                      const int* __restrict__ order, int* __restrict__ status) {
    force_half_body<RDF>(own_blk(), H, cs_start, cs_entries, xo, ts, nn, nbr, dF_f, f_fx, rdf, rec, order, status);
}

// forces from the fixed-point sums into the original atom order
__device__ __forceinline__ void force_half_finalize_body(Blk B, int n, const u64* __restrict__ f_fx, int fstride,
                                                         const int* __restrict__ order, double* __restrict__ f) {
    const int k = B.x * blockDim.x + threadIdx.x;
    if (k >= n) return;
    const int o = order[k];
    f[3 * o] = (double)(long long)f_fx[k] * kForceUnit;
    f[3 * o + 1] = (double)(long long)f_fx[fstride + k] * kForceUnit;
    f[3 * o + 2] = (double)(long long)f_fx[2 * fstride + k] * kForceUnit;
}
__global__ void force_half_finalize_kernel(int n, const u64* __restrict__ f_fx, int fstride,
                                           const int* __restrict__ order, double* __restrict__ f) {
    force_half_finalize_body(own_blk(), n, f_fx, fstride, order, f);
}

// ---------------------------------------------------------------------------
// charge solver: out_X = sum_Y sym_XY v_Y and, with WITH_C, cz_X = chi_X +
// sum_Y Z_Y asym_XY (ctip.f90:85-110, the as-written CTIP_SOLVER forms), once
// per pair: sym is symmetric, asym_XY and asym_YX differ only in the Slater
// exponential of the row atom.

struct CtipHalfTab {
    float ex1x, ex1y;          // -2 xi_X log2(e), -2 xi_Y log2(e)
    float xix, xiy;            // xi_X, xi_Y
    float Sx[4], Sy[2];        // fifj_s = -(eX SX(r) + eY SY(r)) / r
    float ZX, ZY;              // Z_X, Z_Y
};

struct CtipHalfParams {
    float pa, na2l, kc;        // kErfcP a, -a^2 log2(e), kc
    int cap, splits, g0, n;
    float4 sh[kEntries];
    CtipHalfTab tab[4];        // (metal, metal), (metal, O), (O, metal), (O, O)
};

// sym and the two asym Slater parts of two pairs (packed)
template <bool SAME>
__device__ __forceinline__ void ctip_pair_pk(const CtipHalfTab& T, const CtipHalfParams& C, v2 r2, v2& sym,
                                             v2& ax_, v2& ay_) {
    const v2 ir = rsqrt(r2);
    const v2 r = r2 * ir;
    const v2 eX = ex2(r * bc(T.ex1x));
    v2 num = eX * fma2(r, fma2(r, fma2(r, bc(T.Sx[3]), bc(T.Sx[2])), bc(T.Sx[1])), bc(T.Sx[0]));
    v2 eY = eX;
    if (!SAME) {
        eY = ex2(r * bc(T.ex1y));
        num = fma2(eY, fma2(r, bc(T.Sy[1]), bc(T.Sy[0])), num);
    }
    const v2 fifj = bc(-1.f) * num * ir;
    // erfc(a r) = t P(t) exp(-(a r)^2), t = 1 / (1 + kErfcP a r)
    const v2 tt = rcp(fma2(r, bc(C.pa), bc(1.f)));
    const v2 erf_ = tt * erfc_poly(tt) * ex2(r2 * bc(C.na2l));
    sym = bc(C.kc) * fma2(erf_, ir, fifj);
    // kc (afb_X - fifj) and kc (afb_Y - fifj), afb_S = -e_S (xi_S + 1/r)
    ax_ = bc(C.kc) * (bc(-1.f) * eX * (ir + bc(T.xix)) - fifj);
    ay_ = bc(C.kc) * (bc(-1.f) * eY * (ir + bc(T.xiy)) - fifj);
}

template <bool WITH_C, bool TILED, int TI>
__device__ __forceinline__ void ctip_half_batch(const CtipHalfParams& C, const float4* etab,
                                                const float4* __restrict__ rsrc, const double* __restrict__ vsrc,
                                                int lim, unsigned E1, unsigned E2, bool v1, bool v2ok,
                                                const float4& ra, float vXf, const Sink<TILED>& acc, double& sr,
                                                double& cz) {
    const CtipHalfTab& T = C.tab[TI];
    constexpr bool SAME = TI == 0 || TI == 3;
    const float4 t1 = etab[min((int)((E1 >> kSkinCodeShift) & kCodeMask), kEntries - 1)];
    const float4 t2 = etab[min((int)((E2 >> kSkinCodeShift) & kCodeMask), kEntries - 1)];
    int i1 = (int)(E1 & kIdxMask) + __float_as_int(t1.w);
    int i2 = (int)(E2 & kIdxMask) + __float_as_int(t2.w);
    i1 = (unsigned)i1 < (unsigned)lim ? i1 : 0;
    i2 = (unsigned)i2 < (unsigned)lim ? i2 : 0;
    const float4 B1 = rsrc[i1], B2 = rsrc[i2];
    const v2 dx = mk2((ra.x - B1.x) - t1.x, (ra.x - B2.x) - t2.x);
    const v2 dy = mk2((ra.y - B1.y) - t1.y, (ra.y - B2.y) - t2.y);
    const v2 dz = mk2((ra.z - B1.z) - t1.z, (ra.z - B2.z) - t2.z);
    const v2 r2 = fma2(dx, dx, fma2(dy, dy, dz * dz));
    v2 sym, axy, ayx;
    ctip_pair_pk<SAME>(T, C, r2, sym, axy, ayx);
    const v2 sv = sym * bc(vXf * kRhoScale);        // Y's share sym v_X, scaled
    if (v1) {
        sr = fma((double)sym.v.x, vsrc[i1], sr);
        acc.add(0, i1, __float2ll_rn(sv.v.x));
        if (WITH_C) {
            cz += (double)(T.ZY * axy.v.x);
            acc.add(1, i1, __float2ll_rn(T.ZX * ayx.v.x * kRhoScale));
        }
    }
    if (v2ok) {
        sr = fma((double)sym.v.y, vsrc[i2], sr);
        acc.add(0, i2, __float2ll_rn(sv.v.y));
        if (WITH_C) {
            cz += (double)(T.ZY * axy.v.y);
            acc.add(1, i2, __float2ll_rn(T.ZX * ayx.v.y * kRhoScale));
        }
    }
}

template <bool WITH_C, bool TILED>
__device__ __forceinline__ void ctip_half_atoms(const CtipHalfParams& C, const float4* etab,
                                                const float4* __restrict__ rsrc, const double* __restrict__ vsrc,
                                                int lim, int b0, int b1, int a0, int* next,
                                                const float4* __restrict__ frec, const int* __restrict__ ts,
                                                const double* __restrict__ vin, const int2* __restrict__ nn,
                                                const unsigned* __restrict__ nbr, const Sink<TILED>& acc) {
    const int lane = threadIdx.x & 31;
    const int cap = C.cap;
    for (;;) {
        int X = 0;
        if (lane == 0) X = atomicAdd(next, 1);
        X = __shfl_sync(0xffffffffu, X, 0) + b0;
        if (X >= b1) break;
        const float4 ra = frec[X];
        const int sX = ts[X];
        const double vX = vin[X];
        const float vXf = (float)vX;
        const int2 m = nn[X];
        const unsigned* row = nbr + (size_t)X * cap;
        const bool metal = sX == C.g0;
        double sr = 0.0, cz = 0.0;
        if (metal || sX == 3) {
            const int nb0 = (m.x + 63) >> 6, nb = nb0 + ((m.y + 63) >> 6);
            const unsigned pad = ((unsigned)kSelf << kSkinCodeShift) | (unsigned)X;
            // the next batch's entries are loaded before this batch's arithmetic
            auto load = [&](int j, unsigned& a, unsigned& b) {
                const bool g1 = j >= nb0;
                const int kb = (g1 ? j - nb0 : j) << 6, mg = g1 ? m.y : m.x;
                const unsigned* p = g1 ? row + (cap - 1 - kb - lane) : row + kb + lane;
                a = kb + lane < mg ? p[0] : pad;
                b = kb + 32 + lane < mg ? p[g1 ? -32 : 32] : pad;
            };
            unsigned na = pad, nbE = pad;
            if (nb > 0) load(0, na, nbE);
            for (int j = 0; j < nb; j++) {
                const unsigned E1 = na, E2 = nbE;
                if (j + 1 < nb) load(j + 1, na, nbE);
                const bool g1 = j >= nb0;
                const int kb = (g1 ? j - nb0 : j) << 6, mg = g1 ? m.y : m.x;
                const bool v1 = kb + lane < mg, v2ok = kb + 32 + lane < mg;
                if (metal) {
                    if (!g1) ctip_half_batch<WITH_C, TILED, 0>(C, etab, rsrc, vsrc, lim, E1, E2, v1, v2ok, ra, vXf, acc, sr, cz);
                    else ctip_half_batch<WITH_C, TILED, 1>(C, etab, rsrc, vsrc, lim, E1, E2, v1, v2ok, ra, vXf, acc, sr, cz);
                } else {
                    if (!g1) ctip_half_batch<WITH_C, TILED, 2>(C, etab, rsrc, vsrc, lim, E1, E2, v1, v2ok, ra, vXf, acc, sr, cz);
                    else ctip_half_batch<WITH_C, TILED, 3>(C, etab, rsrc, vsrc, lim, E1, E2, v1, v2ok, ra, vXf, acc, sr, cz);
                }
            }
        }
        sr = warp_sum(sr);
        if (WITH_C) cz = warp_sum(cz);
        if (lane == 0) {
            acc.own(0, X, __double2ll_rn(sr * kRhoScaleD));
            if (WITH_C) acc.own(1, X, __double2ll_rn(cz * kRhoScaleD));
        }
    }
}

template <bool WITH_C>
__global__ void __launch_bounds__(kH2Threads, 1)
    ctip_half_kernel(const __grid_constant__ CtipHalfParams C, const int* __restrict__ cs_start,
                     const int* __restrict__ cs_entries, const float4* __restrict__ frec, const int* __restrict__ ts,
                     const int2* __restrict__ nn, const unsigned* __restrict__ nbr, const double* __restrict__ vin,
                     u64* __restrict__ gacc, int gstride) {
    extern __shared__ __align__(16) unsigned char ctip_smem[];
    float4* trec = reinterpret_cast<float4*>(ctip_smem);
    double* tv = reinterpret_cast<double*>(trec + kHCCap);
    unsigned* tlo = reinterpret_cast<unsigned*>(tv + kHCCap);   // [2][cap]
    unsigned* thi = tlo + 2 * kHCCap;                             // [2][cap]
    __shared__ float4 etab[kEntries];
    __shared__ HalfTile T;
    __shared__ int next;
    const int tid = threadIdx.x;
    const int cell = blockIdx.x / C.splits, part = blockIdx.x - cell * C.splits;
    if (tid == 0) next = 0;
    half_tile_setup(T, cs_start, cs_entries, cell);
    const int total = T.off[kHalfCells];
    const int2 br = half_range(T, part, C.splits);
    const int b0 = br.x, b1 = br.y;
    const bool tiled = total <= kHCCap;
    if (tid < kEntries) {
        const float4 o = C.sh[tid];
        const int d = tid < kHalfFirst ? -(1 << 28) : (tiled ? T.off[tid - kHalfFirst] - T.start[tid - kHalfFirst] : 0);
        etab[tid] = make_float4(o.x, o.y, o.z, __int_as_float(d));
    }
    if (tiled) {
        int t = 0;
        for (int i = tid; i < total; i += kH2Threads) {
            while (T.off[t + 1] <= i) t++;
            const int src = T.start[t] + (i - T.off[t]);
            cp_async16(&trec[i], frec + src);
            tv[i] = vin[src];
            tlo[i] = 0u;
            thi[i] = 0u;
            if (WITH_C) {
                tlo[kHCCap + i] = 0u;
                thi[kHCCap + i] = 0u;
            }
        }
        cp_async_commit();
        cp_async_wait<0>();
    }
    __syncthreads();
    const int a0 = T.start[0];
    if (tiled)
        ctip_half_atoms<WITH_C, true>(C, etab, trec, tv, total, b0, b1, a0, &next, frec, ts, vin, nn, nbr,
                                      Sink<true>{tlo, thi, kHCCap, gacc, gstride});
    else
        ctip_half_atoms<WITH_C, false>(C, etab, frec, vin, C.n, b0, b1, a0, &next, frec, ts, vin, nn, nbr,
                                       Sink<false>{gacc, gstride});
    __syncthreads();
    if (tiled) half_tile_flush(T, total, tlo, thi, kHCCap, WITH_C ? 2 : 1, gacc, gstride);
}

// out = fixed-point sums; cconst = chi + the fixed-point asym sums
__global__ void ctip_half_finalize_kernel(int n, const u64* __restrict__ gacc, int gstride,
                                          const int* __restrict__ ts, CtipSpecies S, double* __restrict__ out,
                                          double* __restrict__ cconst) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= n) return;
    out[k] = (double)(long long)gacc[k] * kRhoUnit;
    if (cconst) cconst[k] = S.chi[min(ts[k], 4)] + (double)(long long)gacc[gstride + k] * kRhoUnit;
}

// ---------------------------------------------------------------------------
// FP64 energies of a mixed context on its half list: every listed pair once
// (phi, Ewald real space, CTIP: force.f90:84-98, 101-140), the FP64 density
// of both atoms (X's in registers, Y's into fixed-point sums), then the
// embedding energy from the completed densities.
constexpr int kHEThreads = 128;

__device__ __forceinline__ void energy_half_body(Blk B, const PairParams& P, const PairTab<double>* __restrict__ tab,
                                                 const double4* __restrict__ xq, const int* __restrict__ ts,
                                                 const int2* __restrict__ nn, const unsigned* __restrict__ nbr,
                                                 u64* __restrict__ rho_fx, double* __restrict__ acc,
                                                 int* __restrict__ status) {
    __shared__ PairTab<double> st[kSpecies * kSpecies];
    __shared__ double red[kHEThreads / 32];
    for (int k = threadIdx.x; k < kSpecies * kSpecies; k += blockDim.x) st[k] = tab[k];
    __syncthreads();
    const int lane = threadIdx.x & 31, wpb = blockDim.x >> 5;
    double ep = 0.0, ed = 0.0, ec = 0.0;
    int bad = 0;
    for (int X = B.x * wpb + (threadIdx.x >> 5); X < P.n; X += B.n * wpb) {
        const double4 xa = xq[X];
        const int sX = ts[X];
        const int2 m = nn[X];
        const int mt = m.x + m.y;
        const unsigned* row = nbr + (size_t)X * P.cap;
        double rho = 0.0;
        if (sX < kSpecies) {
            // the next entry's partner data is loaded before this entry's arithmetic
            int Yn = 0, sYn = 0;
            double4 xbn = make_double4(0.0, 0.0, 0.0, 0.0);
            auto fetch = [&](int k) {
                Yn = (int)(row[row_slot(2, k, P.cap, m.x)] & kIdxMask);
                sYn = ts[Yn];
                xbn = xq[Yn];
            };
            if (lane < mt) fetch(lane);
            for (int k = lane; k < mt; k += 32) {
                const int Y = Yn, sY = sYn;
                const double4 xb = xbn;
                if (k + 32 < mt) fetch(k + 32);
                if (sY >= kSpecies) { bad |= ST_UNKNOWN_PAIR; continue; }
                double dx, dy, dz;
                min_image(xa, xb, P, dx, dy, dz);
                const double r = sqrt(__dadd_rn(__dadd_rn(__dmul_rn(dx, dx), __dmul_rn(dy, dy)), __dmul_rn(dz, dz)));
                const PairTab<double>& T = st[sX * kSpecies + sY];
                const double rX = T.d_fe * zhou_val<double>(r, T.d_inv_re, T.d_c, T.d_lam);       // force.f90:84
                rho += rX;
                // a same-species pair: the same density at both atoms (force.f90:85)
                const double rY = sX == sY ? rX : T.e_fe * zhou_val<double>(r, T.e_inv_re, T.e_c, T.e_lam);
                add_fixed(rho_fx + Y, __double2ll_rn(rY * kRhoScaleD));
                pair_energy_fp64(T, r, 1.0 / r, xa.w, xb.w, P.a, ep, ed, ec);
            }
        } else if (mt > 0) {
            bad |= ST_UNKNOWN_PAIR;
        }
        rho = warp_sum(rho);
        if (lane == 0) add_fixed(rho_fx + X, __double2ll_rn(rho * kRhoScaleD));
    }
    if (bad) atomicOr(status, bad);
    block_add<kHEThreads>(ep, acc, A_EPAIR, red);
    block_add<kHEThreads>(ed, acc, A_EDIR, red);
    block_add<kHEThreads>(ec, acc, A_ECTIP, red);
}
__global__ void __launch_bounds__(kHEThreads, 6)
    energy_half_kernel(const __grid_constant__ PairParams P, const PairTab<double>* __restrict__ tab,
                       const double4* __restrict__ xq, const int* __restrict__ ts, const int2* __restrict__ nn,
                       const unsigned* __restrict__ nbr, u64* __restrict__ rho_fx, double* __restrict__ acc,
                       int* __restrict__ status) {
    energy_half_body(own_blk(), P, tab, xq, ts, nn, nbr, rho_fx, acc, status);
}

__device__ __forceinline__ void embed_energy_half_body(Blk B, int n, const int* __restrict__ ts,
                                                       const u64* __restrict__ rho_fx, const EmbedParams& E,
                                                       double* __restrict__ acc, int* __restrict__ status) {
    __shared__ double red[256 / 32];
    double eg = 0.0;
    const int X = B.x * blockDim.x + threadIdx.x;
    if (X < n) {
        double Fe, dF;
        if (embed(E, ts[X], (double)(long long)rho_fx[X] * kRhoUnit, Fe, dF)) atomicOr(status, ST_UNKNOWN_ELEMENT);
        eg = Fe;
    }
    block_add<256>(eg, acc, A_EGROUP, red);
}
__global__ void __launch_bounds__(256)
    embed_energy_half_kernel(int n, const int* __restrict__ ts, const u64* __restrict__ rho_fx,
                             const __grid_constant__ EmbedParams E, double* __restrict__ acc,
                             int* __restrict__ status) {
    embed_energy_half_body(own_blk(), n, ts, rho_fx, E, acc, status);
}

// ---------------------------------------------------------------------------
// host

bool half_path(const simox_ctx* c) { return c->using_skin && c->skin_half; }

static int half_prepare(int device) {
    static std::atomic<bool> done[64] = {};   // contexts may run on several host threads
    if (device >= 0 && device < 64 && done[device].load()) return SIMOX_OK;
    cudaError_t e1 = cudaFuncSetAttribute(force_half_kernel<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kH2Smem);
    cudaError_t e4 = cudaFuncSetAttribute(force_half_kernel<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kH2Smem);
    cudaError_t e2 = cudaFuncSetAttribute(ctip_half_kernel<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kHCSmem);
    cudaError_t e3 = cudaFuncSetAttribute(ctip_half_kernel<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kHCSmem);
    if (e1 != cudaSuccess || e2 != cudaSuccess || e3 != cudaSuccess || e4 != cudaSuccess) return SIMOX_E_CUDA;
    if (device >= 0 && device < 64) done[device] = true;
    return SIMOX_OK;
}

int filter_density_half(simox_ctx* c) {
    if (int st = half_prepare(c->device)) return st;
    Half1Params H;
    std::memset(&H, 0, sizeof(H));
    H.F.pp = pair_params(c);
    H.F.rcut2 = c->rcut2;
    H.F.rcut2f = (float)c->rcut2;
    H.F.band = filter_band(c);
    H.F.nc = make_int3(c->nc[0], c->nc[1], c->nc[2]);
    H.F.cap_s = c->cap_s;
    stencil_shifts(c, H.F.sh);
    H.splits = std::max(1, std::min(16, c->force_splits));
    H.g0 = c->g0_species;
    memset_async(c, c->rho_fx, 0, sizeof(u64) * (size_t)c->n, c->stream);
    if (c->n > 0) {
        Launch L(c, "neighbor_filter_density");
        const int g = c->ncell_s * H.splits;
        launch_k<kH1Threads, 3, filter_half_body>(c, filter_half_kernel, g, 0, c->stream, H, c->tab_f, c->xq_s,
            c->rec_s, c->pair_order, c->cs_start, c->cs_entries, reinterpret_cast<const int2*>(c->nn_s), c->nbr_s,
            reinterpret_cast<int2*>(c->nn), c->nbr, c->rho_fx, c->status, c->nn_max, c->nn_tot);
    }
    if (c->n > 0) {
        Launch L(c, "eam_embed");
        launch_k<256, 1, embed_half_body>(c, embed_half_kernel, (c->n + 255) / 256, 0, c->stream, c->n, c->t_s,
            c->rho_fx, embed_params(c->pot), c->rho_s, c->dF_s, c->dF_f, c->status);
    }
    return check_launch(c);
}

int force_half(simox_ctx* c, bool rdf) {
    if (int st = half_prepare(c->device)) return st;
    PairParams P = pair_params(c);
    Half2Params H;
    std::memset(&H, 0, sizeof(H));
    PackParams& Q = H.Q;
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
    H.lcs = make_double3(c->lcs[0], c->lcs[1], c->lcs[2]);
    H.nc = make_int3(c->nc[0], c->nc[1], c->nc[2]);
    H.splits = std::max(1, std::min(16, c->force_splits));
    H.g0 = g0;
    H.n = c->n;
    H.fstride = c->cap;
    memset_async(c, c->fx_acc, 0, sizeof(u64) * 3 * (size_t)H.fstride, c->stream);
    {
        Launch L(c, "pair_force");
        const int g = c->ncell_s * H.splits;
        if (rdf)
            launch_k<kH2Threads, 1, force_half_body<true>>(c, force_half_kernel<true>, g, kH2Smem, c->stream, H,
                c->cs_start, c->cs_entries, c->xo_s, c->t_s, reinterpret_cast<const int2*>(c->nn), c->nbr, c->dF_f,
                c->fx_acc, c->rdf, c->rec_s, c->pair_order, c->status);
        else
            launch_k<kH2Threads, 1, force_half_body<false>>(c, force_half_kernel<false>, g, kH2Smem, c->stream, H,
                c->cs_start, c->cs_entries, c->xo_s, c->t_s, reinterpret_cast<const int2*>(c->nn), c->nbr, c->dF_f,
                c->fx_acc, c->rdf, c->rec_s, c->pair_order, c->status);
    }
    {
        Launch L(c, "pair_force_finalize");
        launch_k<256, 1, force_half_finalize_body>(c, force_half_finalize_kernel, (c->n + 255) / 256, 0, c->stream,
            c->n, c->fx_acc, H.fstride, c->pair_order, c->f);
    }
    return check_launch(c);
}

int energy_half(simox_ctx* c) {
    memset_async(c, c->rho_fx, 0, sizeof(u64) * (size_t)c->n, c->stream);
    {
        Launch L(c, "pair_energy_fp64");
        const int wpb = kHEThreads / 32;
        const int g = std::max(1, std::min((c->n + wpb - 1) / wpb, num_sms(c) * 12));
        launch_k<kHEThreads, 6, energy_half_body>(c, energy_half_kernel, g, 0, c->stream, pair_params(c), c->tab_d,
            c->xq_s, c->t_s, reinterpret_cast<const int2*>(c->nn), c->nbr, c->rho_fx, c->acc, c->status);
    }
    {
        Launch L(c, "eam_embed_energy");
        launch_k<256, 1, embed_energy_half_body>(c, embed_energy_half_kernel, (c->n + 255) / 256, 0, c->stream, c->n,
            c->t_s, c->rho_fx, embed_params(c->pot), c->acc, c->status);
    }
    return check_launch(c);
}

static CtipHalfTab ctip_half_tab(const simox_potential& P, int X, int Y) {
    CtipHalfTab t;
    std::memset(&t, 0, sizeof(t));
    const double L2E = 1.4426950408889634;
    const simox_potn& pX = P.param[X];
    const simox_potn& pY = P.param[Y];
    t.ex1x = (float)(-2.0 * pX.xi * L2E);
    t.ex1y = (float)(-2.0 * pY.xi * L2E);
    t.xix = (float)pX.xi;
    t.xiy = (float)pY.xi;
    t.ZX = (float)pX.Z;
    t.ZY = (float)pY.Z;
    double Px[5], Py[5], Qx[5], Qy[5], Sx[4], Sy[4];
    ctip_coefs<double>(pX.xi, pY.xi, X == Y, pX.fafb[Y], Px, Py, Qx, Qy, Sx, Sy);
    for (int k = 0; k < 4; k++) t.Sx[k] = (float)Sx[k];
    t.Sy[0] = (float)Sy[0];
    t.Sy[1] = (float)Sy[1];
    return t;
}

static CtipHalfParams ctip_half_params(const simox_ctx* c) {
    CtipHalfParams C;
    std::memset(&C, 0, sizeof(C));
    C.pa = (float)(kErfcP * c->a);
    C.na2l = (float)(-c->a * c->a * 1.4426950408889634);
    C.kc = (float)SX_KC;
    C.cap = c->nnb_cap;
    C.splits = std::max(1, std::min(16, c->force_splits));
    C.g0 = c->g0_species;
    C.n = c->n;
    stencil_shifts(c, C.sh);
    const int g0 = c->g0_species;
    C.tab[0] = ctip_half_tab(c->pot, g0, g0);
    C.tab[1] = ctip_half_tab(c->pot, g0, 3);
    C.tab[2] = ctip_half_tab(c->pot, 3, g0);
    C.tab[3] = ctip_half_tab(c->pot, 3, 3);
    return C;
}

double ctip_half_unit() { return kRhoUnit; }

int ctip_half_launch(simox_ctx* c, const double* vin, cudaStream_t s) {
    if (int st = half_prepare(c->device)) return st;
    const CtipHalfParams C = ctip_half_params(c);
    Launch L(c, "ctip_matvec_pairs");
    ctip_half_kernel<false><<<c->ncell_s * C.splits, kH2Threads, kHCSmem, s>>>(
        C, c->cs_start, c->cs_entries, c->frec_s, c->t_s, reinterpret_cast<const int2*>(c->nn), c->nbr, vin,
        c->fx_acc, c->cap);
    return check_launch(c);
}

int ctip_pair_half(simox_ctx* c, const double* vin, double* out, double* cconst, const CtipSpecies& S) {
    if (int st = half_prepare(c->device)) return st;
    const CtipHalfParams C = ctip_half_params(c);
    const int gstride = c->cap;
    memset_async(c, c->fx_acc, 0, sizeof(u64) * (cconst ? 2 : 1) * (size_t)gstride, c->stream);
    const int g = c->ncell_s * C.splits;
    if (cconst)
        ctip_half_kernel<true><<<g, kH2Threads, kHCSmem, c->stream>>>(C, c->cs_start, c->cs_entries, c->frec_s, c->t_s,
                                                                     reinterpret_cast<const int2*>(c->nn), c->nbr, vin,
                                                                     c->fx_acc, gstride);
    else
        ctip_half_kernel<false><<<g, kH2Threads, kHCSmem, c->stream>>>(C, c->cs_start, c->cs_entries, c->frec_s,
                                                                      c->t_s, reinterpret_cast<const int2*>(c->nn),
                                                                      c->nbr, vin, c->fx_acc, gstride);
    ctip_half_finalize_kernel<<<(c->n + 255) / 256, 256, 0, c->stream>>>(c->n, c->fx_acc, gstride, c->t_s, S, out,
                                                                         cconst);
    return check_launch(c);
}

}  // namespace sx
