// simox_internal.cuh -- device context, pair-parameter tables and helpers of
// the B200 force / charge path.  Internal to libsimox_b200.so.
#pragma once

#include <cuda_runtime.h>
#include <cufft.h>
#include <cstdint>
#include <cstddef>
#include <string>
#include <vector>

#include "simox_gpu.h"

#define SX_KC     14.399644154020082   // datafmt.f90:23
#define SX_TFM    10.180505306645389   // datafmt.f90:24
#define SX_PI     3.1415926535897931   // datafmt.f90:25
#define SX_SQRTPI 1.7724538509055159   // datafmt.f90:26
#define SX_WPEN   20.0                 // datafmt.f90:28 (w)

namespace sx {

constexpr int kSpecies = 4;           // Al, Ni, Fe, O on the device tables (H is rejected)
constexpr int kMaxOrder = 8;
constexpr int kEntries = 27;          // self + 13 forward + 13 reverse stencil cells
// Neighbour-list entry: atom index (bits 0-25) | skin-grid stencil position
// of the partner (bits 26-30, skin mode) | "this atom is the reference's i"
// (bit 31, exact lists).
constexpr unsigned kIsA = 0x80000000u;
constexpr unsigned kIdxMask = 0x03ffffffu;
constexpr unsigned kSkinIdxMask = kIdxMask;
constexpr int kSkinCodeShift = 26;
constexpr unsigned kCodeMask = 31u;

// Device status bits (OR-ed by kernels, read by the host after a call).
enum : int {
    ST_CELL_OVERFLOW = 1, ST_NBR_OVERFLOW = 2, ST_UNKNOWN_PAIR = 4, ST_UNKNOWN_ELEMENT = 8,
    ST_POSITION = 16, ST_UNSUPPORTED = 32, ST_LINE_NOBRACKET = 64,  // Brent: 100 steps without convergence
    ST_RNG = 128,                                                    // thermostat: 100 rejected draws
    ST_SYNC = 256                                                    // a grid-wide wait gave up
};

// Slots of the FP64 accumulator array (energies and reductions).
enum : int {
    A_EPAIR = 0, A_EDIR, A_ECTIP, A_EGROUP, A_EREC, A_FSUM0, A_FSUM1, A_FSUM2,
    A_MV2, A_MV2S0, A_MV2S1 = A_MV2S0 + 1, A_MV2S4 = A_MV2S0 + 4, A_NS0, A_NS4 = A_NS0 + 4,
    // CTIP
    A_GSUM, A_PSUM, A_PMAX, A_GP, A_PAP, A_QSUM, A_Q2SUM, A_ESUM, A_NACT,
    A_LINE0,                    // 32 line-search samples
    A_COUNT = A_LINE0 + 32
};

// Uniform pair table: entry [X][Y] holds everything atom X needs about a
// partner Y.  All EAM forms of eam.f90 used on the Al/Ni/Fe-O path are sums of
// Zhou terms  g(r) = exp(-c (r/re - 1)) / (1 + (r/re - lam)^20).
template <typename R>
struct PairTab {
    // density at X contributed by Y (force.f90:84-85 with eam.f90 fj)
    R d_fe, d_inv_re, d_c, d_lam;
    // density at Y contributed by X
    R e_fe, e_inv_re, e_c, e_lam;
    // pair potential phi = A gA - B gB
    R p_inv_re, p_A, p_alpha, p_kappa, p_B, p_beta, p_lambda;
    // CTIP (force.f90:101-140): xi, Z of X and Y; fifj = -(eX PX(r) + eY PY(r)),
    // dfifj/dr = eX QX(r) + eY QY(r) with P = c0 + c1 r + c2 r^2 + c3 r^3 + cm1/r
    // and Q = d0 + d1 r + d2 r^2 + dm1/r + dm2/r^2; eS = exp(-2 xi_S r).
    R xi_x, xi_y, Z_x, Z_y;
    R Px[5], Py[5], Qx[5], Qy[5];
    // CTIP solver coefficients (ctip.f90:85-110): fifj_s = -(eX SX(r) + eY SY(r))/r
    // with S = s0 + s1 r + s2 r^2 + s3 r^3 (as-written CTIP_SOLVER form).
    R Sx[4], Sy[4];
    int valid;          // 0: the pair form is not on the GPU path
    int pad_;
};

// Slater 1s Coulomb-integral coefficients fafb(a,b,1..4) (datafmt.f90:201-220)
// for the exponents xa of the row species and xb of the column species; same:
// the diagonal form.  T = double, or a dual number for d/dxi.
template <typename T>
inline void slater_fafb(T xa, T xb, bool same, T f[4]) {
    if (same) {
        f[0] = T(1.0);
        f[1] = 11.0 * xa / 8.0;
        f[2] = 0.75 * (xa * xa);
        f[3] = (xa * xa * xa) / 6.0;
    } else {
        const T apb = xa + xb, amb = xa - xb, bma = xb - xa;
        const T a2 = xa * xa, b2 = xb * xb, a4 = a2 * a2, b4 = b2 * b2;
        f[0] = xa * b4 / (apb * apb) / (amb * amb);
        f[1] = xb * a4 / (apb * apb) / (bma * bma);
        f[2] = (3.0 * a2 * b4 - b4 * b2) / (apb * apb * apb) / (amb * amb * amb);
        f[3] = (3.0 * b2 * a4 - a4 * a2) / (apb * apb * apb) / (bma * bma * bma);
    }
}

// CTIP coefficient polynomials of one pair table entry (PairTab Px..Sy) from
// the exponents xx (X), xy (Y) and X's fafb row entry f for Y.  T as above.
template <typename T>
inline void ctip_coefs(T xx, T xy, bool same, const T f[4], T Px[5], T Py[5], T Qx[5], T Qy[5], T Sx[4],
                       T Sy[4]) {
    for (int k = 0; k < 5; k++) Px[k] = Py[k] = Qx[k] = Qy[k] = T(0.0);
    for (int k = 0; k < 4; k++) Sx[k] = Sy[k] = T(0.0);
    if (same) {
        const T xi = xx;
        // fifj = -e (1 + f2 r + f3 r^2 + f4 r^3)              force.f90:107-110
        Px[0] = T(1.0); Px[1] = f[1]; Px[2] = f[2]; Px[3] = f[3];
        // dfifj = e((2xi r+1)(1/r^2+f2/r+f3+f4 r) - (f2/r+2f3+3f4 r)) force.f90:111-118
        Qx[0] = 2.0 * xi * f[1] - f[2]; Qx[1] = 2.0 * xi * f[2] - 2.0 * f[3];
        Qx[2] = 2.0 * xi * f[3]; Qx[3] = 2.0 * xi; Qx[4] = T(1.0);
        // CTIP_SOLVER: -e (1 + xr(f2 + xr(f3 + xr f4)))/r, xr = xi r  ctip.f90:91-93
        Sx[0] = T(1.0); Sx[1] = f[1] * xi; Sx[2] = f[2] * xi * xi; Sx[3] = f[3] * xi * xi * xi;
    } else {
        // fifj = -f1 eX - f2 eY - f3 eX/r - f4 eY/r            force.f90:126-129
        Px[0] = f[0]; Px[4] = f[2];
        Py[0] = f[1]; Py[4] = f[3];
        // dfifj = 2xX f1 eX + 2xY f2 eY + f3 eX(1+2xX r)/r^2 + f4 eY(1+2xY r)/r^2  force.f90:130-133
        Qx[0] = 2.0 * xx * f[0]; Qx[3] = 2.0 * xx * f[2]; Qx[4] = f[2];
        Qy[0] = 2.0 * xy * f[1]; Qy[3] = 2.0 * xy * f[3]; Qy[4] = f[3];
        // CTIP_SOLVER: -eX(f1 + f3/r) - eY(f2 + f4/r)          ctip.f90:97-100
        Sx[0] = f[2]; Sx[1] = f[0];
        Sy[0] = f[3]; Sy[1] = f[1];
    }
}

// Device resources of one PME precision (grid, half spectrum, G/N, plans).
struct PmeRes {
    bool dbl = false, ready = false;
    void* grid = nullptr;       // real grid K1*K2*K3 (x fastest)
    void* cgrid = nullptr;      // half-spectrum complex grid
    void* infl = nullptr;       // G/N on the half spectrum
    unsigned long long* acc = nullptr;   // spread sums, 64-bit fixed point (zero between spreads)
    cufftHandle r2c = 0, c2r = 0;
};

struct Profile {
    std::vector<std::string> names;
    std::vector<double> ms;
    std::vector<long long> launches;
};

}  // namespace sx

namespace sx {
struct AdjointState;
struct Recorder;
}

struct simox_ctx {
    int device = 0;
    cudaStream_t stream = nullptr;      // the stream every entry point issues on
    cudaStream_t side = nullptr;        // md_run: PME overlapped with the pair passes
    cudaEvent_t ev_fork = nullptr, ev_join = nullptr;
    double* f_rec = nullptr;            // reciprocal forces of the overlapped PME (original order)
    simox_setup setup{};
    simox_potential pot{};
    int n = 0, cap = 0;
    int precision = SIMOX_FP64;
    int flags = 0;
    double box[3]{}, inv_box[3]{}, hbox[3]{};
    double rcut = 0, rcut2 = 0, a = 0, dr_rdf = 0;
    int nc[3]{}, ncell = 0;
    double lc[3]{};
    bool fast_cells = false;
    int fft[3]{}, order = 4;
    size_t ngrid = 0, nhalf = 0;
    int npt_max = SIMOX_NPT_MAX, nnb_cap = 1024;
    int force_splits = 1;       // CTAs per skin cell of the mixed pair passes (simox_set_tuning); one
                                // 1024-thread CTA per cell measured fastest at 128k (0.349 ms vs 0.405 at 2)
    unsigned long long md_step_no = 0;   // md_run's current step: the stochastic thermostat's draw counter
    sx::AdjointState* adj = nullptr;   // parameter-adjoint model (simox_set_eam_spline)
    bool adj_warm = false;             // adjoint: refine the held charges by Newton, no CG first
    bool adj_fwd32 = false;            // adjoint: FP32 pair terms in the forward passes
    bool coop_brent = true;            // the charge solver's line search as one cooperative grid
    bool spline_on = false;

    // species present
    bool has_h = false;

    // original-order state
    int* id = nullptr;          // species 1..5
    double* x = nullptr;        // [cap][3]
    double* v = nullptr;
    double* f = nullptr;
    double* q = nullptr;
    double* xm = nullptr;       // per-atom mass (from species)

    // cells
    int* cell_of = nullptr;     // [cap]
    int* cell_xyz = nullptr;    // [cap] packed cell coordinates x | y<<10 | z<<20
    int* cell_count = nullptr;  // [ncell]
    int* cell_start = nullptr;  // [ncell+1]
    int* cell_fill = nullptr;   // [ncell]
    int* sorted = nullptr;      // [cap] original index of sorted slot
    int* pair13 = nullptr;      // [ncell*13] 1-based (reference layout)
    int* entries = nullptr;     // [ncell*27] cell | dir<<28
    std::vector<int> h_pair13;

    // pair-kernel order: the reference cell order (sorted) or, in skin mode,
    // the skin-grid order (perm) that persists between skin-list rebuilds
    int* pair_order = nullptr;
    bool skin_mode = false;     // the box admits the skin list
    bool skin_valid = false;    // perm / x0 / skin list belong to this atom set
    bool using_skin = false;    // the current order is the skin order
    bool skin_half = false;     // the skin list (and the exact list filtered from it) holds each pair once:
                                // mixed precision with one metal species plus oxygen (pair_half.cu)
    bool cells_fresh = false;   // reference cells binned after the last move
    bool in_box = false;        // every coordinate in [-L/2, L/2]
    double skin = 1.0;
    int ncs[3]{}, ncell_s = 0, npt_max_s = 1024, cap_s = 2048;
    double lcs[3]{};
    int* cs_count = nullptr;
    int* cs_start = nullptr;
    int* cs_fill = nullptr;
    int* cs_cell_of = nullptr;
    int* cs_entries = nullptr;
    int* perm = nullptr;
    double* x0 = nullptr;       // positions at the last skin rebuild (original order)
    int* skin_flag = nullptr;   // device: [0] rebuild needed, [1] rebuilds so far
    int* nn_s = nullptr;        // skin list counts (int2)
    unsigned* nbr_s = nullptr;  // skin list rows [cap*cap_s]

    // sorted copies
    double4* xq_s = nullptr;    // x, y, z, q
    int* t_s = nullptr;         // species 0..4
    float4* rec_s = nullptr;    // skin filter record in pair order: skin-cell offset, (cell, species)
    float4* frec_s = nullptr;   // skin force record in pair order: skin-cell offset, charge
    double4* xo_s = nullptr;    // the same offset in FP64 (x, y, z) and the charge (w): the
                                // half-list force pass forms separations from it in FP64
    int g0_species = -1;        // the one non-oxygen species present, or -1
    bool rho_ready = false;     // rho/F' of the filter pass are current (context precision)

    // neighbour list
    int* nn = nullptr;          // [cap] int2: (metal partners, oxygen partners)
    unsigned* nbr = nullptr;    // [cap*nnb_cap]; metal partners from the front, oxygen from the back
    int* nn_max = nullptr;      // device max
    unsigned long long* nn_tot = nullptr;

    // fixed-point accumulators of the half-list passes (pair_half.cu)
    unsigned long long* rho_fx = nullptr;   // [cap] densities, 2^40
    unsigned long long* fx_acc = nullptr;   // [3][cap] forces 2^32, or two charge-solver sums 2^40

    // EAM
    double* rho_s = nullptr;
    double* dF_s = nullptr;
    float* dF_f = nullptr;      // FP32 copy of F' for the mixed pair kernel

    // pair tables
    sx::PairTab<double>* tab_d = nullptr;
    sx::PairTab<float>* tab_f = nullptr;
    sx::PairTab<float> h_tab_f[sx::kSpecies * sx::kSpecies];   // host copy (kernel-parameter tables)

    // PME: pme[0] in the context's precision; pme[1] the FP64 twin that a
    // mixed-precision context uses when energies are requested
    sx::PmeRes pme[2];
    double* psi = nullptr;      // full-grid psi (reference layout)
    double* bmod = nullptr;     // per-dimension 1/|b|^2, K1+K2+K3

    // CTIP
    double* c_const = nullptr;  // chi + sum Z asym (sorted)
    double* g = nullptr;        // -dU/dq (sorted)
    double* pv = nullptr;       // direction (sorted)
    double* Ap = nullptr;       // A p (sorted)
    double* qs = nullptr;       // charges (sorted, FP64)
    double* jp = nullptr;       // J' per sorted atom
    int* act = nullptr;         // active-set indices
    double* line = nullptr;     // line search scalars (bracket, alpha, ...)

    // reductions / status
    double* acc = nullptr;      // [A_COUNT]
    double* h_acc = nullptr;    // pinned mirror
    int* status = nullptr;
    int* h_status = nullptr;    // pinned
    int* rdf = nullptr;         // [SIMOX_RDF_LEN]

    // validity
    bool have_ids = false, cells_valid = false, gathered = false, list_valid = false, psi_valid = false;
    bool cells_listed = false;   // the reference link lists (sorted) belong to the last binning
    bool eam_valid = false;

    // timing / counters
    cudaEvent_t t0 = nullptr, t1 = nullptr;
    bool profiling = false;
    sx::Profile prof;
    std::vector<cudaEvent_t> ev_pool;
    std::vector<std::pair<int, std::pair<cudaEvent_t, cudaEvent_t>>> ev_pending;
    long long launches = 0;

    // md_run: instantiated CUDA graphs of one loop step, keyed by everything
    // that changes the launch sequence; dropped when the atom set changes
    struct StepGraph {
        unsigned long long key = 0;
        double dt = 0.0, T = 0.0;
        cudaGraphExec_t exec = nullptr;
        long long kernels = 0;
    };
    StepGraph graphs[4];
    int graph_next = 0;
    bool graphs_on = true;
    unsigned long long graph_gen = 0;   // bumped whenever captured launches go stale (drop_graphs)
    // set while a batch records this context's step: launches, memsets, event
    // records and waits and FFTs are written down instead of issued
    sx::Recorder* rec = nullptr;
    double eself = 0.0;         // sys%Eself of the last PME_SELF or CTIP_SOLVER
    int last_max_nnb = 0;
    long long last_tot_nnb = 0;
};

// ---------------------------------------------------------------------------
// host-side helpers shared between translation units
namespace sx {

int cuda_status(cudaError_t e);
int check_launch(simox_ctx* c);
int read_status(simox_ctx* c);          // sync + convert device status bits
int profile_id(simox_ctx* c, const char* name);
void prof_begin(simox_ctx* c, int id, cudaEvent_t* a, cudaEvent_t* b);
void prof_end(simox_ctx* c, int id, cudaEvent_t a, cudaEvent_t b);
void prof_collect(simox_ctx* c);
int num_sms(simox_ctx* c);

// RAII-like launch bracket for per-family timing
struct Launch {
    simox_ctx* c; int id; cudaEvent_t a = nullptr, b = nullptr;
    Launch(simox_ctx* c_, const char* name) : c(c_), id(-1) {
        c->launches++;
        if (c->profiling) { id = profile_id(c, name); prof_begin(c, id, &a, &b); }
    }
    ~Launch() { if (id >= 0) prof_end(c, id, a, b); }
};

// cells.cu
int build_cell_tables(simox_ctx* c);
int cell_sort(simox_ctx* c);
int ensure_cell_lists(simox_ctx* c);
int gather_sorted(simox_ctx* c);
int build_list(simox_ctx* c);
int ensure_list(simox_ctx* c);
int ensure_gathered(simox_ctx* c);
int setup_skin(simox_ctx* c);
// pair.cu
int build_pair_tables(simox_ctx* c);
int eam_density(simox_ctx* c, bool eflag);
int filter_density(simox_ctx* c);
int pair_forces(simox_ctx* c, bool eflag, bool rdf);
// pair_half.cu
bool half_path(const simox_ctx* c);
int filter_density_half(simox_ctx* c);
int force_half(simox_ctx* c, bool rdf);
int energy_half(simox_ctx* c);
// pme.cu
int pme_setup(simox_ctx* c);
int pme_free(simox_ctx* c);
int pme_self(simox_ctx* c);
int pme_forces(simox_ctx* c, bool finalize, bool eflag, double* f_store = nullptr);
void pme_bind_stream(simox_ctx* c);
int pme_potential(simox_ctx* c, const double* charges_sorted, double* phi_out, double scale);
int pme_finalize_forces(simox_ctx* c);
int pme_force_charge_adjoint(simox_ctx* c, const double* wt, double* out);
// adjoint.cu
void adjoint_free(simox_ctx* c);
// ctip.cu
struct CtipSpecies {
    double chi[5], Jp[5], qmin[5], qmax[5], Z[5];
};

int ctip_solve(simox_ctx* c, int max_cg, simox_ctip_report* rep, double tol = 1.0e-3);
CtipSpecies ctip_species(const simox_ctx* c);
// The end of one charge-solver matrix-vector product, fused into the PME
// potential gather: Ap = scale phi(p) + J' p + sr (sr from fixed-point sums
// of the half-list pair kernel), the dots g.p and p.Ap, the active set.
struct CtipFinish {
    const int* ts;
    const double* q;
    const double* g;
    const double* pv;
    const unsigned long long* sr_fx;   // sum_Y sym_XY p_Y, fixed point
    double sr_unit;                    // its scale
    double* Ap;
    int* act;
    int* nact;
    double* acc;
    CtipSpecies S;
};
// spread + convolution of qalt (no gather), then the fused gather + finish
int pme_potential_grid(simox_ctx* c, const double* qalt);
int pme_potential_finish(simox_ctx* c, double scale, const CtipFinish& F);
// out = sum_Y sym_XY vin_Y (sorted order); cconst (may be null) = chi + sum_Y Z_Y asym_XY
void ctip_pair(simox_ctx* c, const double* vin, double* out, double* cconst, const CtipSpecies& S);
int ctip_pair_half(simox_ctx* c, const double* vin, double* out, double* cconst, const CtipSpecies& S);
// the half-list pair kernel alone (sums into c->fx_acc, which the caller zeroes) on stream s
int ctip_half_launch(simox_ctx* c, const double* vin, cudaStream_t s);
double ctip_half_unit();
int ctip_alloc(simox_ctx* c);
// integrate.cu
int vv1(simox_ctx* c, double dt, bool reflect);
int vv2(simox_ctx* c, double dt, bool subtract_mean, const double* f_add = nullptr);
int nvt2_berend(simox_ctx* c, double dt, double T_given, bool subtract_mean, const double* f_add = nullptr);
int update_masses(simox_ctx* c);
// md
int md_run(simox_ctx* c, const simox_md_opts* o, int first, int nsteps, simox_energies* e, int* rdf,
           const simox_oxidation* ox = nullptr, int* n_inserted = nullptr);
// oxidation.cu
int remove_rigid_motion(simox_ctx* c);
int oxide_check(simox_ctx* c, int n_o2, double q_crit, int* due);
int new_o2(simox_ctx* c, int n_o2, double z_new, double T_given, unsigned long long seed, unsigned long long event);
void drop_graphs(simox_ctx* c);
int md_step(simox_ctx* c, const simox_md_opts* o, bool sort, bool estep, bool want_rdf);
int vinit_velocities(simox_ctx* c, unsigned long long seed, double T_given);
int nvt1_stoch(simox_ctx* c, double dt, double alpha);
int nvt2_stoch(simox_ctx* c, double dt, double alpha, double T_given, unsigned long long seed,
               unsigned long long step, bool subtract_mean, const double* f_add);

// device helpers -------------------------------------------------------------
__device__ __forceinline__ double warp_sum(double v) {
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}
__device__ __forceinline__ float warp_sumf(float v) {
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}
__device__ __forceinline__ double warp_max(double v) {
    for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
    return v;
}

// Block-wide sum of one double into acc[slot] (one atomic per block).
template <int NT>
__device__ __forceinline__ void block_add(double v, double* acc, int slot, double* sm) {
    v = warp_sum(v);
    const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
    __syncthreads();
    if (l == 0) sm[w] = v;
    __syncthreads();
    if (w == 0) {
        double t = l < NT / 32 ? sm[l] : 0.0;
        t = warp_sum(t);
        if (l == 0 && t != 0.0) atomicAdd(acc + slot, t);
    }
}

// DNINT: round half away from zero (vverlet.f90:92, force.f90:52)
__device__ __forceinline__ double dnint(double x) { return round(x); }

}  // namespace sx

#include "simox_batched.cuh"
