// pme.cu -- PME_SELF (force.f90:467-517), PME (force.f90:364-464) and the
// potential gather of PHI_MESH (ctip.f90:336-396).
//
// The reference spreads charges with order-4 centred B-splines into a
// complex K1xK2xK3 grid, runs two full complex FFTs (FFTE ZFFT3D, +1 with the
// 1/N scale, then -1), multiplies by psi * prod 1/|b|^2 in between, and
// gathers forces from the real part.  Because the charge grid is real and the
// kernel is even, the same result is one real-to-complex transform, the
// multiply on the half spectrum (with 1/N folded in) and one
// complex-to-real transform (cuFFT D2Z/Z2D or R2C/C2R).  The energy
// Epme = N sum_x Q(x) Qfin(x) is evaluated on the half spectrum as
// sum_k G(k)|Q^(k)|^2 (Parseval), fused into the multiply.
//
// Spline order p is a template parameter: p = 4 uses the reference's cubic
// polynomials (force.f90:389-400) term for term, other even orders the
// cardinal B-spline recursion.  Stencil point n of coordinate u is
// INT(u) - p/2 + 1 + n wrapped by MOD (force.f90:404).  The FP64 path rounds
// the spread weight product to single precision before the multiply by q,
// as force.f90:406 / ctip.f90:359 do with a default-kind CMPLX().
#include "simox_internal.cuh"

#include <algorithm>
#include <atomic>
#include <cmath>
#include <type_traits>
#include <vector>

namespace sx {

// ---------------------------------------------------------------------------
// B-spline weights
template <int P>
__device__ __forceinline__ void bspline_w(double u, double* w, double* dw) {
    if constexpr (P == 4) {
        double z = trunc(u) - u + 1.0;
        w[0] = z * z * z / 6.0;
        dw[0] = -3.0 * (z * z) / 6.0;
        z = z + 1.0;
        w[1] = (-3.0 * (z * z * z) + 12.0 * (z * z) - 12.0 * z + 4.0) / 6.0;
        dw[1] = (9.0 * (z * z) - 24.0 * z + 12.0) / 6.0;
        z = z + 1.0;
        w[2] = (3.0 * (z * z * z) - 24.0 * (z * z) + 60.0 * z - 44.0) / 6.0;
        dw[2] = (-9.0 * (z * z) + 48.0 * z - 60.0) / 6.0;
        z = z + 1.0;
        w[3] = (-(z * z * z) + 12.0 * (z * z) - 48.0 * z + 64.0) / 6.0;
        dw[3] = (3.0 * (z * z) - 24.0 * z + 48.0) / 6.0;
    } else {
        const double fr = u - trunc(u);
        double M[P];
#pragma unroll
        for (int k = 0; k < P; k++) M[k] = 0.0;
        M[0] = fr;
        M[1] = 1.0 - fr;
        double dA[P];
#pragma unroll
        for (int n = 3; n <= P; n++) {
            if (n == P) {
#pragma unroll
                for (int k = 0; k < P; k++) dA[k] = (k < P - 1 ? M[k] : 0.0) - (k >= 1 ? M[k - 1] : 0.0);
            }
            const double div = 1.0 / (double)(n - 1);
#pragma unroll
            for (int k = n - 1; k >= 0; k--) {
                const double xk = fr + k;
                const double a1 = k < n - 1 ? M[k] : 0.0;
                const double a0 = k >= 1 ? M[k - 1] : 0.0;
                M[k] = (xk * a1 + ((double)n - xk) * a0) * div;
            }
        }
#pragma unroll
        for (int s = 0; s < P; s++) { w[s] = M[P - 1 - s]; dw[s] = dA[P - 1 - s]; }
    }
}

struct PmeParams {
    int3 K;
    double3 box;
    double3 kx;      // K/L
    double cst;      // kc N / (V pi)
    int n;
};

__device__ __forceinline__ int wrapi(int v, int K) {
    v %= K;
    return v < 0 ? v + K : v;
}

// Spread: grid[x + K1(y + K2 z)] = sum q W, summed exactly in 64-bit fixed
// point (2^48 units), so the grid does not depend on the order of the adds.
// Atoms are stored cell by cell (skin cells or reference cells), and one CTA
// takes one cell: it finds the box of grid points its atoms' stencils cover
// (unwrapped indices), adds q W there in shared memory -- each 64-bit sum
// held as two 32-bit words with the carry of the low word added into the high
// one -- and then adds the box to the global 64-bit grid `acc` (wrapped), one
// global atomic per touched point instead of one per atom and stencil point.
// A cell whose box exceeds the patch adds straight into `acc`.  A second
// kernel converts `acc` to the grid's type and clears it for the next spread.
// Measured at 128k corundum (PME 128^3, order 6): 38 us for the shared adds,
// about 50 us with the global merge and the conversion.
//
// Per point the work is one FP64 multiply (q scale wx) * (wy wz) and one FP64
// add: RN(x) as an integer is read from the bits of x + 1.5 2^52, the
// magic-number rounding, exact for |x| < 2^51 (|q W| < 8); larger values take
// the conversion instruction.  The FP64 grid keeps the reference's product
// order (wx wy) wz, rounded to FP32 as force.f90:406 does, times q.
constexpr int SP_THREADS = 256;
constexpr int SP_CAP = 9216;                              // patch points: 72 KB, three CTAs per SM
constexpr double kSpreadScale = 281474976710656.0;        // 2^48
constexpr double kSpreadUnit = 1.0 / 281474976710656.0;
constexpr double kMagic = 6755399441055744.0;             // 1.5 2^52

__device__ __forceinline__ long long spread_fixed(double x) {
    return fabs(x) < 2251799813685248.0 ? __double_as_longlong(x + kMagic) - __double_as_longlong(kMagic)
                                        : __double2ll_rn(x);
}

__device__ __forceinline__ void patch_add(unsigned* lo, unsigned* hi, int i, long long v) {
    const unsigned vl = (unsigned)v, vh = (unsigned)((unsigned long long)v >> 32);
    const unsigned old = atomicAdd(lo + i, vl);
    atomicAdd(hi + i, vh + ((unsigned)(old + vl) < old ? 1u : 0u));
}

// x = q W scaled, W = wx wy wz: the reference's FP32-rounded product order on
// the FP64 grid, (q scale wx) (wy wz) otherwise
template <bool ROUND>
__device__ __forceinline__ double spread_term(double q, double qwx, double wx, double wy, double wz, double wyz) {
    if constexpr (ROUND) return q * (double)(float)(wx * wy * wz) * kSpreadScale;
    else return qwx * wyz;
}

// an atom of a cell whose box exceeds the patch: straight into the global sums
template <typename R, int P>
__device__ __noinline__ void spread_atom_global(const PmeParams& S, double q, const double* wx, const double* wy,
                                                const double* wz, int bx, int by, int bz,
                                                unsigned long long* __restrict__ acc) {
    constexpr bool ROUND = sizeof(R) == 8;
    const double qs = q * kSpreadScale;
    for (int c = 0; c < P; c++) {
        const size_t gz = (size_t)wrapi(bz + c, S.K.z) * S.K.y;
        for (int b = 0; b < P; b++) {
            const size_t gyz = (gz + wrapi(by + b, S.K.y)) * S.K.x;
            const double wyz = wy[b] * wz[c];
            for (int aa = 0; aa < P; aa++)
                atomicAdd(acc + gyz + wrapi(bx + aa, S.K.x),
                          (unsigned long long)spread_fixed(spread_term<ROUND>(q, wx[aa] * qs, wx[aa], wy[b], wz[c], wyz)));
        }
    }
}

// The periodic image of grid base b nearest to ref.  The atoms of one cell
// lie within a third of the box of each other (at least three cells per
// axis), but VV_NVE1 wraps an atom that crossed a face of the box to the
// opposite face: taken as is, its base would stretch the cell's patch over
// the whole grid and send the cell to the global-atomics path.
__device__ __forceinline__ int near_image(int b, int ref, int K) {
    const int d = b - ref;
    return d > K / 2 ? b - K : (d < -(K / 2) ? b + K : b);
}

template <typename R, int P>
__device__ __forceinline__ void spread_patch_body(Blk B, const PmeParams& S, const double4* __restrict__ xq,
                                                  const double* __restrict__ qalt, const int* __restrict__ ranges,
                                                  unsigned long long* __restrict__ acc) {
    constexpr bool ROUND = sizeof(R) == 8;   // FP64 grid: the reference's FP32 weight products
    extern __shared__ unsigned sp_words[];  // [SP_CAP] low words, [SP_CAP] high words
    __shared__ int lo3[3], hi3[3], ref3[3];
    const int a0 = ranges[B.x], a1 = ranges[B.x + 1];
    if (a1 <= a0) return;
    const int tid = threadIdx.x;
    if (tid < 3) {
        lo3[tid] = 0x7fffffff;
        hi3[tid] = -0x7fffffff;
        // bases are taken at the image nearest to the cell's first atom
        const double4 a = xq[a0];
        const double x = tid == 0 ? a.x : (tid == 1 ? a.y : a.z);
        const double L = tid == 0 ? S.box.x : (tid == 1 ? S.box.y : S.box.z);
        const int K = tid == 0 ? S.K.x : (tid == 1 ? S.K.y : S.K.z);
        ref3[tid] = __double2int_rz((double)K * (x + L * 0.5) / L) - P / 2 + 1;
    }
    __syncthreads();
    const int Kd[3] = {S.K.x, S.K.y, S.K.z};
    int mn[3] = {0x7fffffff, 0x7fffffff, 0x7fffffff}, mx[3] = {-0x7fffffff, -0x7fffffff, -0x7fffffff};
    for (int k = a0 + tid; k < a1; k += SP_THREADS) {
        const double4 a = xq[k];
        const double q = qalt ? qalt[k] : a.w;
        if (q == 0.0) continue;
        const double u[3] = {(double)S.K.x * (a.x + S.box.x * 0.5) / S.box.x,
                             (double)S.K.y * (a.y + S.box.y * 0.5) / S.box.y,
                             (double)S.K.z * (a.z + S.box.z * 0.5) / S.box.z};
#pragma unroll
        for (int d = 0; d < 3; d++) {
            const int b = near_image(__double2int_rz(u[d]) - P / 2 + 1, ref3[d], Kd[d]);
            mn[d] = min(mn[d], b);
            mx[d] = max(mx[d], b);
        }
    }
#pragma unroll
    for (int d = 0; d < 3; d++) {
        for (int o = 16; o > 0; o >>= 1) {
            mn[d] = min(mn[d], __shfl_xor_sync(0xffffffffu, mn[d], o));
            mx[d] = max(mx[d], __shfl_xor_sync(0xffffffffu, mx[d], o));
        }
        if ((tid & 31) == 0) {
            atomicMin(&lo3[d], mn[d]);
            atomicMax(&hi3[d], mx[d]);
        }
    }
    __syncthreads();
    if (hi3[0] < lo3[0]) return;   // no charged atom
    const int ex = hi3[0] - lo3[0] + P, ey = hi3[1] - lo3[1] + P, ez = hi3[2] - lo3[2] + P;
    const bool tiled = (long long)ex * ey * ez <= SP_CAP;
    unsigned* plo = sp_words;
    unsigned* phi = sp_words + SP_CAP;
    if (tiled) {
        for (int i = tid; i < ex * ey * ez; i += SP_THREADS) {
            plo[i] = 0u;
            phi[i] = 0u;
        }
        __syncthreads();
    }
    for (int k = a0 + tid; k < a1; k += SP_THREADS) {
        const double4 a = xq[k];
        const double q = qalt ? qalt[k] : a.w;
        if (q == 0.0) continue;
        double wx[P], wy[P], wz[P], d[P];
        const double ux = (double)S.K.x * (a.x + S.box.x * 0.5) / S.box.x;
        const double uy = (double)S.K.y * (a.y + S.box.y * 0.5) / S.box.y;
        const double uz = (double)S.K.z * (a.z + S.box.z * 0.5) / S.box.z;
        bspline_w<P>(ux, wx, d);
        bspline_w<P>(uy, wy, d);
        bspline_w<P>(uz, wz, d);
        const int bx = near_image(__double2int_rz(ux) - P / 2 + 1, ref3[0], Kd[0]);
        const int by = near_image(__double2int_rz(uy) - P / 2 + 1, ref3[1], Kd[1]);
        const int bz = near_image(__double2int_rz(uz) - P / 2 + 1, ref3[2], Kd[2]);
        if (!tiled) {
            spread_atom_global<R, P>(S, q, wx, wy, wz, bx, by, bz, acc);
            continue;
        }
        const double qs = q * kSpreadScale;
        double qwx[P];
#pragma unroll
        for (int aa = 0; aa < P; aa++) qwx[aa] = ROUND ? 0.0 : wx[aa] * qs;
        const int rx = bx - lo3[0], ry = by - lo3[1], rz = bz - lo3[2];
#pragma unroll
        for (int c = 0; c < P; c++) {
#pragma unroll
            for (int b = 0; b < P; b++) {
                const int row = ((rz + c) * ey + (ry + b)) * ex + rx;
                const double wyz = ROUND ? 0.0 : wy[b] * wz[c];
#pragma unroll
                for (int aa = 0; aa < P; aa++)
                    patch_add(plo, phi, row + aa, spread_fixed(spread_term<ROUND>(q, qwx[aa], wx[aa], wy[b], wz[c], wyz)));
            }
        }
    }
    if (!tiled) return;
    __syncthreads();
    const int warp = tid >> 5, lane = tid & 31;
    for (int rowi = warp; rowi < ey * ez; rowi += SP_THREADS / 32) {
        const int iy = rowi % ey, iz = rowi / ey;
        const size_t gyz = ((size_t)wrapi(lo3[2] + iz, S.K.z) * S.K.y + wrapi(lo3[1] + iy, S.K.y)) * S.K.x;
        for (int ix = lane; ix < ex; ix += 32) {
            const int i = rowi * ex + ix;
            const unsigned long long v = ((unsigned long long)phi[i] << 32) | plo[i];
            if (v) atomicAdd(acc + gyz + wrapi(lo3[0] + ix, S.K.x), v);
        }
    }
}
template <typename R, int P>
__global__ void __launch_bounds__(SP_THREADS, sizeof(R) == 8 ? 2 : 3)
    spread_patch_kernel(const __grid_constant__ PmeParams S, const double4* __restrict__ xq,
                        const double* __restrict__ qalt, const int* __restrict__ ranges,
                        unsigned long long* __restrict__ acc) {
    spread_patch_body<R, P>(own_blk(), S, xq, qalt, ranges, acc);
}

// grid = acc in the grid's type; acc cleared for the next spread
template <typename R>
__device__ __forceinline__ void spread_convert_body(Blk B, size_t n, unsigned long long* __restrict__ acc,
                                                    R* __restrict__ grid) {
    const size_t i = B.x * (size_t)blockDim.x + threadIdx.x;
    if (i >= n) return;
    grid[i] = (R)((double)(long long)acc[i] * kSpreadUnit);
    acc[i] = 0ull;
}
template <typename R>
__global__ void spread_convert_kernel(size_t n, unsigned long long* __restrict__ acc, R* __restrict__ grid) {
    spread_convert_body<R>(own_blk(), n, acc, grid);
}

// half-spectrum multiply by G/N and energy sum_k G |Q^|^2 (Hermitian weights)
template <typename R>
__device__ __forceinline__ void influence_body(Blk B, size_t nhalf, int kx_half, int K1,
                                               typename std::conditional<sizeof(R) == 8, double2,
                                               float2>::type* __restrict__ cg, const R* __restrict__ infl,
                                               double Ngrid, double* __restrict__ acc, int eflag) {
    __shared__ double red[256 / 32];
    double e = 0.0;
    for (size_t i = (size_t)B.x * blockDim.x + threadIdx.x; i < nhalf; i += (size_t)B.n * blockDim.x) {
        const int kx = (int)(i % kx_half);
        auto c = cg[i];
        const R g = infl[i];
        if (eflag) {
            const double wgt = (kx == 0 || (2 * kx == K1)) ? 1.0 : 2.0;
            e += wgt * (double)g * ((double)c.x * (double)c.x + (double)c.y * (double)c.y);
        }
        c.x *= g;
        c.y *= g;
        cg[i] = c;
    }
    if (eflag) block_add<256>(e * Ngrid, acc, A_EREC, red);
}
template <typename R>
__global__ void __launch_bounds__(256)
    influence_kernel(size_t nhalf, int kx_half, int K1, typename std::conditional<sizeof(R) == 8, double2,
                     float2>::type* __restrict__ cg, const R* __restrict__ infl, double Ngrid,
                     double* __restrict__ acc, int eflag) {
    influence_body<R>(own_blk(), nhalf, kx_half, K1, cg, infl, Ngrid, acc, eflag);
}

// gather forces: f[o] += -cst q sum (dW_x W_y W_z kx, ...) Qfin  (force.f90:439-456)
template <typename R, int P>
__device__ __forceinline__ void gather_force_body(Blk B, const PmeParams& S, const double4* __restrict__ xq,
                                                  const R* __restrict__ grid, const int* __restrict__ sorted,
                                                  double* __restrict__ f, double* __restrict__ acc, int store) {
    __shared__ double red[128 / 32];
    const int k = B.x * blockDim.x + threadIdx.x;
    double fo[3] = {0.0, 0.0, 0.0};
    if (k < S.n) {
        const double4 a = xq[k];
        double wx[P], wy[P], wz[P], dx[P], dy[P], dz[P];
        const double ux = (double)S.K.x * (a.x + S.box.x * 0.5) / S.box.x;
        const double uy = (double)S.K.y * (a.y + S.box.y * 0.5) / S.box.y;
        const double uz = (double)S.K.z * (a.z + S.box.z * 0.5) / S.box.z;
        bspline_w<P>(ux, wx, dx);
        bspline_w<P>(uy, wy, dy);
        bspline_w<P>(uz, wz, dz);
        const int bx = __double2int_rz(ux) - P / 2 + 1;
        const int by = __double2int_rz(uy) - P / 2 + 1;
        const int bz = __double2int_rz(uz) - P / 2 + 1;
        int ix[P];
#pragma unroll
        for (int s = 0; s < P; s++) ix[s] = wrapi(bx + s, S.K.x);
        double sx = 0.0, sy = 0.0, sz = 0.0;
#pragma unroll
        for (int c = 0; c < P; c++) {
            const size_t gz = (size_t)wrapi(bz + c, S.K.z) * S.K.y;
#pragma unroll
            for (int b = 0; b < P; b++) {
                const size_t gyz = (gz + wrapi(by + b, S.K.y)) * S.K.x;
                R tx = 0, tw = 0;
#pragma unroll
                for (int aa = 0; aa < P; aa++) {
                    const R g = grid[gyz + ix[aa]];
                    tx += (R)dx[aa] * g;
                    tw += (R)wx[aa] * g;
                }
                sx += (double)tx * wy[b] * wz[c];
                sy += (double)tw * dy[b] * wz[c];
                sz += (double)tw * wy[b] * dz[c];
            }
        }
        const double pre = -S.cst * a.w;
        fo[0] = pre * sx * S.kx.x;
        fo[1] = pre * sy * S.kx.y;
        fo[2] = pre * sz * S.kx.z;
        const int o = sorted[k];
        if (store) {   // separate reciprocal-force buffer
            f[3 * o] = fo[0];
            f[3 * o + 1] = fo[1];
            f[3 * o + 2] = fo[2];
        } else {
            f[3 * o] += fo[0];
            f[3 * o + 1] += fo[1];
            f[3 * o + 2] += fo[2];
        }
    }
    block_add<128>(fo[0], acc, A_FSUM0, red);
    block_add<128>(fo[1], acc, A_FSUM1, red);
    block_add<128>(fo[2], acc, A_FSUM2, red);
}
template <typename R, int P>
__global__ void __launch_bounds__(128)
    gather_force_kernel(const __grid_constant__ PmeParams S, const double4* __restrict__ xq,
                        const R* __restrict__ grid, const int* __restrict__ sorted, double* __restrict__ f,
                        double* __restrict__ acc, int store) {
    gather_force_body<R, P>(own_blk(), S, xq, grid, sorted, f, acc, store);
}

// gather potential: phi[k] = scale * sum W Qfin  (ctip.f90:381-393)
template <typename R, int P>
__global__ void __launch_bounds__(128)
    gather_pot_kernel(PmeParams S, const double4* __restrict__ xq, const R* __restrict__ grid,
                      double* __restrict__ phi, double scale) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= S.n) return;
    const double4 a = xq[k];
    double wx[P], wy[P], wz[P], d[P];
    const double ux = (double)S.K.x * (a.x + S.box.x * 0.5) / S.box.x;
    const double uy = (double)S.K.y * (a.y + S.box.y * 0.5) / S.box.y;
    const double uz = (double)S.K.z * (a.z + S.box.z * 0.5) / S.box.z;
    bspline_w<P>(ux, wx, d);
    bspline_w<P>(uy, wy, d);
    bspline_w<P>(uz, wz, d);
    const int bx = __double2int_rz(ux) - P / 2 + 1;
    const int by = __double2int_rz(uy) - P / 2 + 1;
    const int bz = __double2int_rz(uz) - P / 2 + 1;
    int ix[P];
#pragma unroll
    for (int s = 0; s < P; s++) ix[s] = wrapi(bx + s, S.K.x);
    double sum = 0.0;
#pragma unroll
    for (int c = 0; c < P; c++) {
        const size_t gz = (size_t)wrapi(bz + c, S.K.z) * S.K.y;
#pragma unroll
        for (int b = 0; b < P; b++) {
            const size_t gyz = (gz + wrapi(by + b, S.K.y)) * S.K.x;
            R tw = 0;
#pragma unroll
            for (int aa = 0; aa < P; aa++) tw += (R)wx[aa] * grid[gyz + ix[aa]];
            sum += (double)tw * wy[b] * wz[c];
        }
    }
    phi[k] = scale * sum;
}

// The potential gather of PHI_MESH (ctip.f90:381-393) fused with the end of
// the charge solver's matrix-vector product: Ap = scale phi(p) + J' p + sr,
// the dots g.p and p.Ap and the atoms whose charge can cross a bound for a
// step in [-1, 1] (the Brent line search's active set).
template <typename R, int P>
__global__ void __launch_bounds__(128)
    gather_pot_ctip_kernel(PmeParams S, const double4* __restrict__ xq, const R* __restrict__ grid, double scale,
                           CtipFinish F) {
    __shared__ double red[128 / 32];
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    double gp = 0.0, pap = 0.0;
    if (k < S.n) {
        const double4 a = xq[k];
        double wx[P], wy[P], wz[P], d[P];
        const double ux = (double)S.K.x * (a.x + S.box.x * 0.5) / S.box.x;
        const double uy = (double)S.K.y * (a.y + S.box.y * 0.5) / S.box.y;
        const double uz = (double)S.K.z * (a.z + S.box.z * 0.5) / S.box.z;
        bspline_w<P>(ux, wx, d);
        bspline_w<P>(uy, wy, d);
        bspline_w<P>(uz, wz, d);
        const int bx = __double2int_rz(ux) - P / 2 + 1;
        const int by = __double2int_rz(uy) - P / 2 + 1;
        const int bz = __double2int_rz(uz) - P / 2 + 1;
        int ix[P];
#pragma unroll
        for (int s = 0; s < P; s++) ix[s] = wrapi(bx + s, S.K.x);
        double sum = 0.0;
#pragma unroll
        for (int c = 0; c < P; c++) {
            const size_t gz = (size_t)wrapi(bz + c, S.K.z) * S.K.y;
#pragma unroll
            for (int b = 0; b < P; b++) {
                const size_t gyz = (gz + wrapi(by + b, S.K.y)) * S.K.x;
                R tw = 0;
#pragma unroll
                for (int aa = 0; aa < P; aa++) tw += (R)wx[aa] * grid[gyz + ix[aa]];
                sum += (double)tw * wy[b] * wz[c];
            }
        }
        const int sp = min(F.ts[k], 4);
        const double p = F.pv[k];
        const double sr = (double)(long long)F.sr_fx[k] * F.sr_unit;
        const double ap = scale * sum + F.S.Jp[sp] * p + sr;
        F.Ap[k] = ap;
        gp = F.g[k] * p;
        pap = p * ap;
        const double qi = F.q[k], ab = fabs(p);
        if (qi - ab < F.S.qmin[sp] || qi + ab > F.S.qmax[sp]) F.act[atomicAdd(F.nact, 1)] = k;
    }
    block_add<128>(gp, F.acc, A_GP, red);
    block_add<128>(pap, F.acc, A_PAP, red);
}

// psi(m) = exp(-pi^2 m2/a^2)/m2, m = 0 -> 0   (force.f90:500-514)
__global__ void psi_kernel(int3 K, double3 box, double a2, double* __restrict__ psi) {
    const size_t N = (size_t)K.x * K.y * K.z;
    for (size_t g = (size_t)blockIdx.x * blockDim.x + threadIdx.x; g < N; g += (size_t)gridDim.x * blockDim.x) {
        int i = (int)(g % K.x), j = (int)((g / K.x) % K.y), k = (int)(g / ((size_t)K.x * K.y));
        int ix = (i + K.x / 2) % K.x - K.x / 2;
        int iy = (j + K.y / 2) % K.y - K.y / 2;
        int iz = (k + K.z / 2) % K.z - K.z / 2;
        int m = ix * ix + iy * iy + iz * iz;
        double v = 0.0;
        if (m != 0) {
            double m2 = (double)(ix * ix) / (box.x * box.x) + (double)(iy * iy) / (box.y * box.y) +
                        (double)(iz * iz) / (box.z * box.z);
            v = exp(-m2 * (SX_PI * SX_PI) / a2) / m2;
        }
        psi[g] = v;
    }
}

template <typename R>
__global__ void infl_build_kernel(int3 K, int kxh, const double* __restrict__ psi, const double* __restrict__ bm,
                                  double invN, R* __restrict__ infl) {
    const size_t N = (size_t)kxh * K.y * K.z;
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < N; i += (size_t)gridDim.x * blockDim.x) {
        int kx = (int)(i % kxh), ky = (int)((i / kxh) % K.y), kz = (int)(i / ((size_t)kxh * K.y));
        double p = psi[kx + (size_t)K.x * (ky + (size_t)K.y * kz)];
        infl[i] = (R)(p * bm[kx] * bm[K.x + ky] * bm[K.x + K.y + kz] * invN);
    }
}

// self energy (force.f90:486-498)
__global__ void self_energy_kernel(int n, const int* __restrict__ id, const double* __restrict__ q,
                                   const double* __restrict__ chi, const double* __restrict__ J,
                                   const double* __restrict__ qmin, const double* __restrict__ qmax,
                                   double* __restrict__ acc) {
    __shared__ double red[256 / 32];
    double q2 = 0.0, es = 0.0;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        double qi = q[i];
        int s = id[i] - 1;
        q2 -= qi * qi;
        es += chi[s] * qi + 0.5 * J[s] * (qi * qi);
        double dq = qi - qmin[s];
        if (dq < 0.0) es += 2.0 * SX_WPEN * (dq * dq);
        dq = qi - qmax[s];
        if (dq > 0.0) es += 2.0 * SX_WPEN * (dq * dq);
    }
    block_add<256>(q2, acc, A_Q2SUM, red);
    block_add<256>(es, acc, A_ESUM, red);
}

// ---------------------------------------------------------------------------
// host side
static double bmod_inv_host(int p, int k, int K) {
    double th = 2.0 * SX_PI * (double)k / (double)K;
    if (p == 4) {
        double z = 4.0 + 2.0 * cos(th);
        return 36.0 / (z * z);     // 36 / (4 + 2cos)^2 of force.f90:415-420
    }
    // centred B-spline values beta(t) = M_p(t + p/2) at integer t
    std::vector<double> M(p + 1, 0.0), Mn(p + 1, 0.0);
    M[0] = 0.0; M[1] = 1.0;                 // M_2 at 0, 1 (fr = 0)
    for (int n = 3; n <= p; n++) {
        for (int kk = 0; kk < n; kk++) {
            double a1 = kk < n - 1 ? M[kk] : 0.0, a0 = kk >= 1 ? M[kk - 1] : 0.0;
            Mn[kk] = (kk * a1 + (n - kk) * a0) / (double)(n - 1);
        }
        for (int kk = 0; kk < n; kk++) M[kk] = Mn[kk];
    }
    double b = 0.0;                          // M[kk] = M_p(kk)
    for (int kk = 1; kk < p; kk++) b += M[kk] * cos(th * (kk - p / 2));
    return 1.0 / (b * b);
}

static void pme_res_free(PmeRes& R) {
    if (R.ready) {
        cufftDestroy(R.r2c);
        cufftDestroy(R.c2r);
    }
    cudaFree(R.grid); cudaFree(R.cgrid); cudaFree(R.infl); cudaFree(R.acc);
    R = PmeRes();
}

int pme_free(simox_ctx* c) {
    pme_res_free(c->pme[0]);
    pme_res_free(c->pme[1]);
    cudaFree(c->psi); cudaFree(c->bmod);
    c->psi = c->bmod = nullptr;
    return SIMOX_OK;
}

static int pme_res_init(simox_ctx* c, PmeRes& R, bool dbl) {
    const int* K = c->fft;
    const size_t rs = dbl ? sizeof(double) : sizeof(float);
    R.dbl = dbl;
    if (cudaMalloc(&R.grid, c->ngrid * rs) != cudaSuccess) return SIMOX_E_NOMEM;
    if (cudaMalloc(&R.cgrid, c->nhalf * 2 * rs) != cudaSuccess) return SIMOX_E_NOMEM;
    if (cudaMalloc(&R.infl, c->nhalf * rs) != cudaSuccess) return SIMOX_E_NOMEM;
    if (cudaMalloc(&R.acc, c->ngrid * sizeof(unsigned long long)) != cudaSuccess) return SIMOX_E_NOMEM;
    if (cudaMemset(R.acc, 0, c->ngrid * sizeof(unsigned long long)) != cudaSuccess) return SIMOX_E_NOMEM;
    // cuFFT plans: dims slowest-first (K3, K2, K1); K1 is the contiguous x axis
    if (cufftPlan3d(&R.r2c, K[2], K[1], K[0], dbl ? CUFFT_D2Z : CUFFT_R2C) != CUFFT_SUCCESS) return SIMOX_E_FFT_SIZE;
    if (cufftPlan3d(&R.c2r, K[2], K[1], K[0], dbl ? CUFFT_Z2D : CUFFT_C2R) != CUFFT_SUCCESS) {
        cufftDestroy(R.r2c);
        return SIMOX_E_FFT_SIZE;
    }
    cufftSetStream(R.r2c, c->stream);
    cufftSetStream(R.c2r, c->stream);
    R.ready = true;
    return SIMOX_OK;
}

int pme_setup(simox_ctx* c) {
    const int* K = c->fft;
    c->ngrid = (size_t)K[0] * K[1] * K[2];
    c->nhalf = (size_t)(K[0] / 2 + 1) * K[1] * K[2];
    int st = pme_res_init(c, c->pme[0], c->precision == SIMOX_FP64);
    if (st) return st;
    if (c->precision != SIMOX_FP64 && (st = pme_res_init(c, c->pme[1], true))) return st;
    if (cudaMalloc(&c->psi, c->ngrid * sizeof(double)) != cudaSuccess) return SIMOX_E_NOMEM;
    if (cudaMalloc(&c->bmod, (K[0] + K[1] + K[2]) * sizeof(double)) != cudaSuccess) return SIMOX_E_NOMEM;
    std::vector<double> bm(K[0] + K[1] + K[2]);
    int o = 0;
    for (int d = 0; d < 3; d++)
        for (int k = 0; k < K[d]; k++) bm[o++] = bmod_inv_host(c->order, k, K[d]);
    if (cudaMemcpyAsync(c->bmod, bm.data(), bm.size() * sizeof(double), cudaMemcpyHostToDevice, c->stream) !=
        cudaSuccess)
        return SIMOX_E_CUDA;
    return cuda_status(cudaStreamSynchronize(c->stream));
}

// PME_SELF: psi table, influence function(s), self energy into acc
int pme_self(simox_ctx* c) {
    int3 K = make_int3(c->fft[0], c->fft[1], c->fft[2]);
    double3 box = make_double3(c->box[0], c->box[1], c->box[2]);
    {
        Launch L(c, "pme_psi");
        psi_kernel<<<num_sms(c) * 4, 256, 0, c->stream>>>(K, box, c->a * c->a, c->psi);
    }
    const double invN = 1.0 / (double)c->ngrid;
    for (int k = 0; k < 2; k++) {
        PmeRes& R = c->pme[k];
        if (!R.ready) continue;
        Launch L(c, "pme_influence_build");
        if (R.dbl)
            infl_build_kernel<double><<<num_sms(c) * 4, 256, 0, c->stream>>>(K, K.x / 2 + 1, c->psi, c->bmod, invN,
                                                                             (double*)R.infl);
        else
            infl_build_kernel<float><<<num_sms(c) * 4, 256, 0, c->stream>>>(K, K.x / 2 + 1, c->psi, c->bmod, invN,
                                                                            (float*)R.infl);
    }
    c->psi_valid = true;
    if (c->n > 0) {
        // species parameter columns in device scratch (acc tail not used): small uploads
        double h[4][5];
        for (int s = 0; s < 5; s++) {
            h[0][s] = c->pot.param[s].chi; h[1][s] = c->pot.param[s].J;
            h[2][s] = c->pot.param[s].qmin; h[3][s] = c->pot.param[s].qmax;
        }
        double* d = c->line;   // line-search scratch is free outside CTIP
        cudaMemcpyAsync(d, h, sizeof(h), cudaMemcpyHostToDevice, c->stream);
        Launch L(c, "pme_self_energy");
        self_energy_kernel<<<num_sms(c), 256, 0, c->stream>>>(c->n, c->id, c->q, d, d + 5, d + 10, d + 15, c->acc);
    }
    return check_launch(c);
}

template <typename R, int P>
static bool spread_ready(int device) {
    static std::atomic<bool> done[64] = {};   // contexts may run on several host threads
    if (device < 0 || device >= 64) return false;
    if (!done[device].load())
        done[device] = cudaFuncSetAttribute(spread_patch_kernel<R, P>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                            (int)(2 * SP_CAP * sizeof(unsigned))) == cudaSuccess;
    return done[device].load();
}

// one CTA per cell of the atom order (skin cells or reference cells)
template <typename R, int P>
static int run_spread(simox_ctx* c, PmeRes& Rs, const PmeParams& S, const double* qalt) {
    if (!spread_ready<R, P>(c->device)) return SIMOX_E_CUDA;
    Launch L(c, "pme_spread");
    if (c->n > 0) {
        const bool skin = c->using_skin && c->pair_order == c->perm;
        const int* ranges = skin ? c->cs_start : c->cell_start;
        const int nr = skin ? c->ncell_s : c->ncell;
        launch_k<SP_THREADS, sizeof(R) == 8 ? 2 : 3, spread_patch_body<R, P>>(c, spread_patch_kernel<R, P>, nr,
            2 * SP_CAP * sizeof(unsigned), c->stream, S, c->xq_s, qalt, ranges, Rs.acc);
    }
    launch_k<256, 1, spread_convert_body<R>>(c, spread_convert_kernel<R>, (unsigned)((c->ngrid + 255) / 256), 0,
        c->stream, c->ngrid, Rs.acc, (R*)Rs.grid);
    return check_launch(c);
}

// an FFT of a recorded step: written down for the batch to issue
static void record_fft(simox_ctx* c, cufftHandle plan, int kind, void* in, void* out) {
    RecOp op;
    op.kind = RecOp::FFT;
    op.lane = c->rec->lane(c->stream);
    op.plan = plan;
    op.fft = kind;
    op.in = in;
    op.out = out;
    c->rec->ops.push_back(std::move(op));
}

static int run_convolution(simox_ctx* c, PmeRes& Rs, bool eflag) {
    cufftResult r = CUFFT_SUCCESS;
    if (c->rec) record_fft(c, Rs.r2c, Rs.dbl ? 2 : 0, Rs.grid, Rs.cgrid);
    else {
        Launch L(c, "pme_fft_r2c");
        if (Rs.dbl) r = cufftExecD2Z(Rs.r2c, (cufftDoubleReal*)Rs.grid, (cufftDoubleComplex*)Rs.cgrid);
        else r = cufftExecR2C(Rs.r2c, (cufftReal*)Rs.grid, (cufftComplex*)Rs.cgrid);
    }
    if (r != CUFFT_SUCCESS) return SIMOX_E_CUDA;
    {
        Launch L(c, "pme_influence");
        int kxh = c->fft[0] / 2 + 1;
        const int g = (int)std::min<size_t>((size_t)num_sms(c) * 4, (c->nhalf + 255) / 256);
        if (Rs.dbl)
            launch_k<256, 1, influence_body<double>>(c, influence_kernel<double>, g, 0, c->stream, c->nhalf, kxh,
                c->fft[0], (double2*)Rs.cgrid, (const double*)Rs.infl, (double)c->ngrid, c->acc, eflag ? 1 : 0);
        else
            launch_k<256, 1, influence_body<float>>(c, influence_kernel<float>, g, 0, c->stream, c->nhalf, kxh,
                c->fft[0], (float2*)Rs.cgrid, (const float*)Rs.infl, (double)c->ngrid, c->acc, eflag ? 1 : 0);
    }
    if (c->rec) record_fft(c, Rs.c2r, Rs.dbl ? 3 : 1, Rs.cgrid, Rs.grid);
    else {
        Launch L(c, "pme_fft_c2r");
        if (Rs.dbl) r = cufftExecZ2D(Rs.c2r, (cufftDoubleComplex*)Rs.cgrid, (cufftDoubleReal*)Rs.grid);
        else r = cufftExecC2R(Rs.c2r, (cufftComplex*)Rs.cgrid, (cufftReal*)Rs.grid);
    }
    if (r != CUFFT_SUCCESS) return SIMOX_E_CUDA;
    return SIMOX_OK;
}

static PmeParams pme_params(const simox_ctx* c) {
    PmeParams S;
    S.K = make_int3(c->fft[0], c->fft[1], c->fft[2]);
    S.box = make_double3(c->box[0], c->box[1], c->box[2]);
    S.kx = make_double3(c->fft[0] / c->box[0], c->fft[1] / c->box[1], c->fft[2] / c->box[2]);
    double V = c->box[0] * c->box[1] * c->box[2];
    S.cst = SX_KC * (double)c->fft[0] * (double)c->fft[1] * (double)c->fft[2] / V / SX_PI;
    S.n = c->n;
    return S;
}

template <typename R, int P>
static int pme_forces_t(simox_ctx* c, PmeRes& Rs, bool eflag, double* f_store) {
    PmeParams S = pme_params(c);
    int st = run_spread<R, P>(c, Rs, S, nullptr);
    if (!st) st = run_convolution(c, Rs, eflag);
    if (st) return st;
    Launch L(c, "pme_gather_force");
    launch_k<128, 1, gather_force_body<R, P>>(c, gather_force_kernel<R, P>, (S.n + 127) / 128, 0, c->stream, S,
        c->xq_s, (const R*)Rs.grid, c->pair_order, f_store ? f_store : c->f, c->acc, f_store ? 1 : 0);
    return SIMOX_OK;
}

template <typename R, int P>
static int pme_pot_t(simox_ctx* c, PmeRes& Rs, const double* qalt, double* phi, double scale) {
    PmeParams S = pme_params(c);
    int st = run_spread<R, P>(c, Rs, S, qalt);
    if (!st) st = run_convolution(c, Rs, false);
    if (st) return st;
    Launch L(c, "pme_gather_pot");
    gather_pot_kernel<R, P><<<(S.n + 127) / 128, 128, 0, c->stream>>>(S, c->xq_s, (const R*)Rs.grid, phi, scale);
    return SIMOX_OK;
}

// mean-force removal (force.f90:457-460)
__global__ void subtract_mean_kernel(int n, double* __restrict__ f, const double* __restrict__ acc) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    // Fsum(:) = Fsum(:)/DBLE(Npt_all); ff = ff - Fsum   (force.f90:457-459)
    f[3 * i] = __dsub_rn(f[3 * i], __ddiv_rn(acc[A_FSUM0], (double)n));
    f[3 * i + 1] = __dsub_rn(f[3 * i + 1], __ddiv_rn(acc[A_FSUM1], (double)n));
    f[3 * i + 2] = __dsub_rn(f[3 * i + 2], __ddiv_rn(acc[A_FSUM2], (double)n));
}

// cuFFT plans follow the context's current stream
void pme_bind_stream(simox_ctx* c) {
    for (PmeRes& R : c->pme)
        if (R.ready) {
            cufftSetStream(R.r2c, c->stream);
            cufftSetStream(R.c2r, c->stream);
        }
}

int pme_finalize_forces(simox_ctx* c) {
    if (c->n == 0) return SIMOX_OK;
    Launch L(c, "pme_mean_force");
    subtract_mean_kernel<<<(c->n + 255) / 256, 256, 0, c->stream>>>(c->n, c->f, c->acc);
    return check_launch(c);
}

// f_store: write the reciprocal forces there instead of adding them to f
int pme_forces(simox_ctx* c, bool finalize, bool eflag, double* f_store) {
    if (!c->psi_valid) return SIMOX_E_STATE;
    if (int st0 = ensure_gathered(c)) return st0;
    if (c->n == 0) return SIMOX_OK;
    memset_async(c, c->acc + A_FSUM0, 0, 3 * sizeof(double), c->stream);
    int st;
    // energies are FP64: a mixed context uses its FP64 twin when they are requested
    PmeRes& Rs = (eflag && c->pme[1].ready) ? c->pme[1] : c->pme[0];
    const bool dbl = Rs.dbl;
    switch (c->order) {
        case 4: st = dbl ? pme_forces_t<double, 4>(c, Rs, eflag, f_store) : pme_forces_t<float, 4>(c, Rs, eflag, f_store); break;
        case 6: st = dbl ? pme_forces_t<double, 6>(c, Rs, eflag, f_store) : pme_forces_t<float, 6>(c, Rs, eflag, f_store); break;
        case 8: st = dbl ? pme_forces_t<double, 8>(c, Rs, eflag, f_store) : pme_forces_t<float, 8>(c, Rs, eflag, f_store); break;
        default: return SIMOX_E_ARG;
    }
    if (st) return st;
    if (finalize) {
        st = pme_finalize_forces(c);
        if (st) return st;
    }
    return check_launch(c);
}

// ---------------------------------------------------------------------------
// Charge adjoint of the PME forces (FP64 grids).  With a weight field w on
// the atoms (mean already removed, as the mean-force subtraction of
// force.f90:455-460 requires), S = sum_i w_i . F_i^rec and
// F_i^rec = -cst q_i g_i, g_i = grad of the interpolated (G*Q) at x_i, so
//   dS/dq_m = -cst [ w_m . g_m + sum_grid W~_m (G*D) ],
//   D(grid) = sum_i q_i w_i . grad W_i(grid),
// W~ the spread weights (rounded to single precision as the spread rounds
// them, force.f90:406) and grad W the unrounded weight derivatives that the
// force gather uses.
template <int P>
__global__ void __launch_bounds__(128)
    field_dot_kernel(PmeParams S, const double4* __restrict__ xq, const double* __restrict__ grid,
                     const double* __restrict__ wt, double* __restrict__ out, double scale) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= S.n) return;
    const double4 a = xq[k];
    double wx[P], wy[P], wz[P], dx[P], dy[P], dz[P];
    const double ux = (double)S.K.x * (a.x + S.box.x * 0.5) / S.box.x;
    const double uy = (double)S.K.y * (a.y + S.box.y * 0.5) / S.box.y;
    const double uz = (double)S.K.z * (a.z + S.box.z * 0.5) / S.box.z;
    bspline_w<P>(ux, wx, dx);
    bspline_w<P>(uy, wy, dy);
    bspline_w<P>(uz, wz, dz);
    const int bx = __double2int_rz(ux) - P / 2 + 1;
    const int by = __double2int_rz(uy) - P / 2 + 1;
    const int bz = __double2int_rz(uz) - P / 2 + 1;
    double sx = 0.0, sy = 0.0, sz = 0.0;
    for (int c = 0; c < P; c++) {
        const size_t gz = (size_t)wrapi(bz + c, S.K.z) * S.K.y;
        for (int b = 0; b < P; b++) {
            const size_t gyz = (gz + wrapi(by + b, S.K.y)) * S.K.x;
            for (int aa = 0; aa < P; aa++) {
                const double g = grid[gyz + wrapi(bx + aa, S.K.x)];
                sx += dx[aa] * wy[b] * wz[c] * g;
                sy += wx[aa] * dy[b] * wz[c] * g;
                sz += wx[aa] * wy[b] * dz[c] * g;
            }
        }
    }
    out[k] += scale * (wt[3 * k] * sx * S.kx.x + wt[3 * k + 1] * sy * S.kx.y + wt[3 * k + 2] * sz * S.kx.z);
}

template <int P>
__global__ void __launch_bounds__(128)
    spread_dipole_kernel(PmeParams S, const double4* __restrict__ xq, const double* __restrict__ wt,
                         double* __restrict__ grid) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= S.n) return;
    const double4 a = xq[k];
    if (a.w == 0.0) return;
    double wx[P], wy[P], wz[P], dx[P], dy[P], dz[P];
    const double ux = (double)S.K.x * (a.x + S.box.x * 0.5) / S.box.x;
    const double uy = (double)S.K.y * (a.y + S.box.y * 0.5) / S.box.y;
    const double uz = (double)S.K.z * (a.z + S.box.z * 0.5) / S.box.z;
    bspline_w<P>(ux, wx, dx);
    bspline_w<P>(uy, wy, dy);
    bspline_w<P>(uz, wz, dz);
    const int bx = __double2int_rz(ux) - P / 2 + 1;
    const int by = __double2int_rz(uy) - P / 2 + 1;
    const int bz = __double2int_rz(uz) - P / 2 + 1;
    const double px = a.w * wt[3 * k] * S.kx.x, py = a.w * wt[3 * k + 1] * S.kx.y, pz = a.w * wt[3 * k + 2] * S.kx.z;
    for (int c = 0; c < P; c++) {
        const size_t gz = (size_t)wrapi(bz + c, S.K.z) * S.K.y;
        for (int b = 0; b < P; b++) {
            const size_t gyz = (gz + wrapi(by + b, S.K.y)) * S.K.x;
            for (int aa = 0; aa < P; aa++) {
                const double v = px * dx[aa] * wy[b] * wz[c] + py * wx[aa] * dy[b] * wz[c] + pz * wx[aa] * wy[b] * dz[c];
                atomicAdd(grid + gyz + wrapi(bx + aa, S.K.x), v);
            }
        }
    }
}

template <int P>
__global__ void __launch_bounds__(128)
    gather_rounded_kernel(PmeParams S, const double4* __restrict__ xq, const double* __restrict__ grid,
                          double* __restrict__ out, double scale) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= S.n) return;
    const double4 a = xq[k];
    double wx[P], wy[P], wz[P], d[P];
    const double ux = (double)S.K.x * (a.x + S.box.x * 0.5) / S.box.x;
    const double uy = (double)S.K.y * (a.y + S.box.y * 0.5) / S.box.y;
    const double uz = (double)S.K.z * (a.z + S.box.z * 0.5) / S.box.z;
    bspline_w<P>(ux, wx, d);
    bspline_w<P>(uy, wy, d);
    bspline_w<P>(uz, wz, d);
    const int bx = __double2int_rz(ux) - P / 2 + 1;
    const int by = __double2int_rz(uy) - P / 2 + 1;
    const int bz = __double2int_rz(uz) - P / 2 + 1;
    double sum = 0.0;
    for (int c = 0; c < P; c++) {
        const size_t gz = (size_t)wrapi(bz + c, S.K.z) * S.K.y;
        for (int b = 0; b < P; b++) {
            const size_t gyz = (gz + wrapi(by + b, S.K.y)) * S.K.x;
            for (int aa = 0; aa < P; aa++)
                sum += (double)(float)(wx[aa] * wy[b] * wz[c]) * grid[gyz + wrapi(bx + aa, S.K.x)];
        }
    }
    out[k] += scale * sum;
}

template <int P>
static int force_charge_adjoint_t(simox_ctx* c, PmeRes& Rs, const double* wt, double* out) {
    PmeParams S = pme_params(c);
    const int nb = (S.n + 127) / 128;
    int st = run_spread<double, P>(c, Rs, S, nullptr);
    if (!st) st = run_convolution(c, Rs, false);
    if (st) return st;
    {
        Launch L(c, "adjoint_pme_field");
        field_dot_kernel<P><<<nb, 128, 0, c->stream>>>(S, c->xq_s, (const double*)Rs.grid, wt, out, -S.cst);
    }
    cudaMemsetAsync(Rs.grid, 0, c->ngrid * sizeof(double), c->stream);
    {
        Launch L(c, "adjoint_pme_dipole_spread");
        spread_dipole_kernel<P><<<nb, 128, 0, c->stream>>>(S, c->xq_s, wt, (double*)Rs.grid);
    }
    if ((st = run_convolution(c, Rs, false))) return st;
    Launch L(c, "adjoint_pme_dipole_gather");
    gather_rounded_kernel<P><<<nb, 128, 0, c->stream>>>(S, c->xq_s, (const double*)Rs.grid, out, -S.cst);
    return check_launch(c);
}

// out (sorted order) += dS/dq for S = sum_i wt_i . F_i^rec (FP64 context)
int pme_force_charge_adjoint(simox_ctx* c, const double* wt, double* out) {
    if (!c->psi_valid) return SIMOX_E_STATE;
    if (c->n == 0) return SIMOX_OK;
    PmeRes& Rs = c->pme[0];
    if (!Rs.dbl) return SIMOX_E_UNSUPPORTED;
    switch (c->order) {
        case 4: return force_charge_adjoint_t<4>(c, Rs, wt, out);
        case 6: return force_charge_adjoint_t<6>(c, Rs, wt, out);
        case 8: return force_charge_adjoint_t<8>(c, Rs, wt, out);
        default: return SIMOX_E_ARG;
    }
}

// CTIP's PME potential runs on the FP64 grid in both precision modes: with
// the FP32 grid the charges of the reference's nonlinear CG drift by ~3e-6 e
// over a thousand iterations (measured on 500-600 atom Al/O systems), above
// the 1e-6 e bar; the FP64 grid keeps them within 3e-7 e.
int pme_potential(simox_ctx* c, const double* qalt, double* phi, double scale) {
    if (!c->psi_valid) return SIMOX_E_STATE;
    if (c->n == 0) return SIMOX_OK;
    PmeRes& Rs = c->pme[1].ready ? c->pme[1] : c->pme[0];
    const bool dbl = Rs.dbl;
    int st;
    switch (c->order) {
        case 4: st = dbl ? pme_pot_t<double, 4>(c, Rs, qalt, phi, scale) : pme_pot_t<float, 4>(c, Rs, qalt, phi, scale); break;
        case 6: st = dbl ? pme_pot_t<double, 6>(c, Rs, qalt, phi, scale) : pme_pot_t<float, 6>(c, Rs, qalt, phi, scale); break;
        case 8: st = dbl ? pme_pot_t<double, 8>(c, Rs, qalt, phi, scale) : pme_pot_t<float, 8>(c, Rs, qalt, phi, scale); break;
        default: return SIMOX_E_ARG;
    }
    if (st) return st;
    return check_launch(c);
}

template <typename R, int P>
static int pme_grid_t(simox_ctx* c, PmeRes& Rs, const double* qalt) {
    PmeParams S = pme_params(c);
    if (int st = run_spread<R, P>(c, Rs, S, qalt)) return st;
    return run_convolution(c, Rs, false);
}

int pme_potential_grid(simox_ctx* c, const double* qalt) {
    if (!c->psi_valid) return SIMOX_E_STATE;
    if (c->n == 0) return SIMOX_OK;
    PmeRes& Rs = c->pme[1].ready ? c->pme[1] : c->pme[0];
    int st;
    switch (c->order) {
        case 4: st = Rs.dbl ? pme_grid_t<double, 4>(c, Rs, qalt) : pme_grid_t<float, 4>(c, Rs, qalt); break;
        case 6: st = Rs.dbl ? pme_grid_t<double, 6>(c, Rs, qalt) : pme_grid_t<float, 6>(c, Rs, qalt); break;
        case 8: st = Rs.dbl ? pme_grid_t<double, 8>(c, Rs, qalt) : pme_grid_t<float, 8>(c, Rs, qalt); break;
        default: return SIMOX_E_ARG;
    }
    return st ? st : check_launch(c);
}

template <typename R, int P>
static void finish_t(simox_ctx* c, PmeRes& Rs, double scale, const CtipFinish& F) {
    PmeParams S = pme_params(c);
    gather_pot_ctip_kernel<R, P><<<(S.n + 127) / 128, 128, 0, c->stream>>>(S, c->xq_s, (const R*)Rs.grid, scale, F);
}

int pme_potential_finish(simox_ctx* c, double scale, const CtipFinish& F) {
    if (c->n == 0) return SIMOX_OK;
    PmeRes& Rs = c->pme[1].ready ? c->pme[1] : c->pme[0];
    Launch L(c, "ctip_matvec_finish");
    switch (c->order) {
        case 4: Rs.dbl ? finish_t<double, 4>(c, Rs, scale, F) : finish_t<float, 4>(c, Rs, scale, F); break;
        case 6: Rs.dbl ? finish_t<double, 6>(c, Rs, scale, F) : finish_t<float, 6>(c, Rs, scale, F); break;
        case 8: Rs.dbl ? finish_t<double, 8>(c, Rs, scale, F) : finish_t<float, 8>(c, Rs, scale, F); break;
        default: return SIMOX_E_ARG;
    }
    return check_launch(c);
}

}  // namespace sx
