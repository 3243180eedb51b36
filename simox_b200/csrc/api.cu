// api.cu -- the extern "C" boundary declared in include/simox_gpu.h, the
// device context, status handling, profiling and the device-resident loop.
#include "simox_internal.cuh"

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <new>

namespace sx {

int cuda_status(cudaError_t e) {
    if (e == cudaSuccess) return SIMOX_OK;
    if (e == cudaErrorMemoryAllocation) return SIMOX_E_NOMEM;
    if (e == cudaErrorNoDevice || e == cudaErrorInsufficientDriver) return SIMOX_E_NO_DEVICE;
    return SIMOX_E_CUDA;
}

int check_launch(simox_ctx*) { return cuda_status(cudaGetLastError()); }

int read_status(simox_ctx* c) {
    cudaError_t e = cudaMemcpyAsync(c->h_status, c->status, sizeof(int), cudaMemcpyDeviceToHost, c->stream);
    if (e != cudaSuccess) return cuda_status(e);
    e = cudaStreamSynchronize(c->stream);
    if (e != cudaSuccess) return cuda_status(e);
    int s = *c->h_status;
    if (s) cudaMemsetAsync(c->status, 0, sizeof(int), c->stream);
    if (s & ST_POSITION) return SIMOX_E_POSITION;
    if (s & ST_CELL_OVERFLOW) return SIMOX_E_CELL_OVERFLOW;
    if (s & ST_NBR_OVERFLOW) return SIMOX_E_NBR_OVERFLOW;
    if (s & ST_UNKNOWN_PAIR) return SIMOX_E_UNKNOWN_PAIR;
    if (s & ST_UNKNOWN_ELEMENT) return SIMOX_E_UNKNOWN_ELEMENT;
    if (s & ST_UNSUPPORTED) return SIMOX_E_UNSUPPORTED;
    if (s & ST_LINE_NOBRACKET) return SIMOX_E_BRENT;
    if (s & ST_RNG) return SIMOX_E_RNG;
    if (s & ST_SYNC) return SIMOX_E_SYNC;
    return SIMOX_OK;
}

int num_sms(simox_ctx* c) {
    static int cached_dev = -1, cached = 148;
    if (cached_dev != c->device) {
        int v = 0;
        if (cudaDeviceGetAttribute(&v, cudaDevAttrMultiProcessorCount, c->device) == cudaSuccess && v > 0) cached = v;
        cached_dev = c->device;
    }
    return cached;
}

int profile_id(simox_ctx* c, const char* name) {
    for (size_t i = 0; i < c->prof.names.size(); i++)
        if (c->prof.names[i] == name) return (int)i;
    c->prof.names.emplace_back(name);
    c->prof.ms.push_back(0.0);
    c->prof.launches.push_back(0);
    return (int)c->prof.names.size() - 1;
}

static cudaEvent_t pool_event(simox_ctx* c) {
    if (!c->ev_pool.empty()) {
        cudaEvent_t e = c->ev_pool.back();
        c->ev_pool.pop_back();
        return e;
    }
    cudaEvent_t e = nullptr;
    cudaEventCreate(&e);
    return e;
}

void prof_begin(simox_ctx* c, int, cudaEvent_t* a, cudaEvent_t* b) {
    *a = pool_event(c);
    *b = pool_event(c);
    cudaEventRecord(*a, c->stream);
}

void prof_end(simox_ctx* c, int id, cudaEvent_t a, cudaEvent_t b) {
    cudaEventRecord(b, c->stream);
    c->ev_pending.push_back({id, {a, b}});
    if (c->ev_pending.size() > 4096) prof_collect(c);
}

void prof_collect(simox_ctx* c) {
    if (c->ev_pending.empty()) return;
    cudaStreamSynchronize(c->stream);
    if (c->side) cudaStreamSynchronize(c->side);
    for (auto& p : c->ev_pending) {
        float ms = 0.f;
        if (cudaEventElapsedTime(&ms, p.second.first, p.second.second) == cudaSuccess) c->prof.ms[p.first] += ms;
        c->prof.launches[p.first] += 1;
        c->ev_pool.push_back(p.second.first);
        c->ev_pool.push_back(p.second.second);
    }
    c->ev_pending.clear();
}

// ---------------------------------------------------------------------------
// device-resident main loop (main.f90:40-84 with TAG_SET main.f90:376-414)

// PME forces into f_rec on c->side, forked from c->stream; ev_join marks
// their end.  With the per-launch profile on, PME stays on c->stream so that
// each launch's event span holds that launch alone, not the time it shared
// the SMs with the concurrent pair passes.
static int pme_fork(simox_ctx* c, bool estep) {
    if (c->profiling) {
        const int st = pme_forces(c, false, estep, c->f_rec);
        event_record(c, c->ev_join, c->stream);
        return st;
    }
    event_record(c, c->ev_fork, c->stream);
    stream_wait(c, c->side, c->ev_fork);
    std::swap(c->stream, c->side);
    pme_bind_stream(c);
    const int st = pme_forces(c, false, estep, c->f_rec);
    std::swap(c->stream, c->side);
    pme_bind_stream(c);
    if (st) return st;
    event_record(c, c->ev_join, c->side);
    return SIMOX_OK;
}

// One step without CTIP: VV_NVE1 (or VV_NVT1_STOCH), CELL_SORT, FORCE (+ PME
// on the side stream), VV_NVE2 / VV_NVT2_BEREND / VV_NVT2_STOCH.  Every launch goes to c->stream or, for
// PME, to c->side forked from and joined back to it, so the whole step can be
// captured into one CUDA graph.
int md_step(simox_ctx* c, const simox_md_opts* o, bool sort, bool estep, bool want_rdf) {
    int st;
    if (estep) memset_async(c, c->acc, 0, sizeof(double) * (A_EREC + 1), c->stream);
    const bool stoch = o->thermostat && o->thermo_stoch;
    if ((st = stoch ? nvt1_stoch(c, o->dt, o->alpha) : vv1(c, o->dt, o->reflect != 0))) return st;
    if (sort && (st = cell_sort(c))) return st;
    // PME (positions and charges only) runs on the side stream while the
    // pair passes run; its forces land in f_rec and the second half kick
    // adds them: f = f_pair + f_rec - Fsum/N, as FORCE + PME would leave f.
    if ((st = ensure_gathered(c))) return st;
    if ((st = pme_fork(c, estep))) return st;
    if ((st = ensure_list(c))) return st;
    if ((st = eam_density(c, estep))) return st;
    if ((st = pair_forces(c, estep, want_rdf))) return st;
    stream_wait(c, c->stream, c->ev_join);
    if (stoch) st = nvt2_stoch(c, o->dt, o->alpha, o->T_given, o->seed, c->md_step_no, true, c->f_rec);
    else if (o->thermostat) st = nvt2_berend(c, o->dt, o->T_given, true, c->f_rec);
    else st = vv2(c, o->dt, true, c->f_rec);
    return st;
}

void drop_graphs(simox_ctx* c) {
    c->graph_gen++;   // graphs of a batch that hold this context's launches are stale too
    for (auto& g : c->graphs) {
        if (g.exec) cudaGraphExecDestroy(g.exec);
        g = simox_ctx::StepGraph{};
    }
}

// The step as a graph: captured on first use of its key, then replayed.
// A capture that fails (an API call the capture does not allow) turns graphs
// off for this context and the step runs eagerly.
static int md_step_graph(simox_ctx* c, const simox_md_opts* o, bool sort, bool estep, bool want_rdf) {
    const unsigned long long key = 1ull | (sort ? 2ull : 0) | (estep ? 4ull : 0) | (want_rdf ? 8ull : 0) |
                                   (o->reflect ? 16ull : 0) | (o->thermostat ? 32ull : 0) |
                                   ((unsigned long long)(unsigned)c->n << 32);
    simox_ctx::StepGraph* hit = nullptr;
    for (auto& g : c->graphs)
        if (g.exec && g.key == key && g.dt == o->dt && g.T == o->T_given) hit = &g;
    if (!hit) {
        cudaGraph_t graph = nullptr;
        if (cudaStreamBeginCapture(c->stream, cudaStreamCaptureModeThreadLocal) != cudaSuccess) {
            c->graphs_on = false;
            return md_step(c, o, sort, estep, want_rdf);
        }
        const long long l0 = c->launches;
        int st = md_step(c, o, sort, estep, want_rdf);
        const cudaError_t ce = cudaStreamEndCapture(c->stream, &graph);
        cudaGetLastError();
        cudaGraphExec_t exec = nullptr;
        if (st || ce != cudaSuccess || !graph || cudaGraphInstantiate(&exec, graph, 0) != cudaSuccess) {
            if (graph) cudaGraphDestroy(graph);
            cudaGetLastError();
            c->graphs_on = false;
            if (st) return st;
            // the capture recorded nothing that ran: run the step eagerly
            c->launches = l0;
            return md_step(c, o, sort, estep, want_rdf);
        }
        cudaGraphDestroy(graph);
        simox_ctx::StepGraph& g = c->graphs[c->graph_next];
        c->graph_next = (c->graph_next + 1) % 4;
        if (g.exec) cudaGraphExecDestroy(g.exec);
        g.key = key;
        g.dt = o->dt;
        g.T = o->T_given;
        g.exec = exec;
        g.kernels = c->launches - l0;
        c->launches = l0;
        hit = &g;
    }
    c->launches += hit->kernels;
    return cuda_status(cudaGraphLaunch(hit->exec, c->stream));
}

int md_run(simox_ctx* c, const simox_md_opts* o, int first, int nsteps, simox_energies* e, int* rdf,
           const simox_oxidation* ox, int* n_inserted) {
    if (!c->psi_valid || !c->cells_valid) return SIMOX_E_STATE;
    const bool want_rdf = rdf != nullptr || o->accumulate_rdf;
    if (want_rdf) cudaMemsetAsync(c->rdf, 0, sizeof(int) * SIMOX_RDF_LEN, c->stream);
    int st = SIMOX_OK;
    for (int step = first; step < first + nsteps; step++) {
        c->md_step_no = (unsigned long long)step;
        const bool new_charge = o->freq_new > 0 && (o->charge_every_step || step % o->freq_new == 1);
        const bool sort = o->freq_sort > 0 && step % o->freq_sort == 0;
        const bool estep = o->freq_stat <= 0 || step % o->freq_stat == 0;   // TAG_SET status rule
        if (new_charge) {
            // CTIP_SOLVER between CELL_SORT and FORCE: eager (host-driven CG)
            if (estep) cudaMemsetAsync(c->acc, 0, sizeof(double) * (A_EREC + 1), c->stream);
            const bool stoch = o->thermostat && o->thermo_stoch;
            if ((st = stoch ? nvt1_stoch(c, o->dt, o->alpha) : vv1(c, o->dt, o->reflect != 0))) return st;
            if (sort && (st = cell_sort(c))) return st;
            if (ox) {
                // oxidation mode (main.f90:69-74): REMOVE_RIGID_MOTION, OXIDE_CHECK
                // and, when due, NEW_O2, all on the device; the moved and the new
                // atoms are binned again before the charge solve
                if ((st = remove_rigid_motion(c))) return st;
                int due = 0;
                if ((st = oxide_check(c, ox->n_o2, ox->q_crit, &due))) return st;
                if (due && ox->n_o2 > 0) {
                    if ((st = new_o2(c, ox->n_o2, ox->z_new, o->T_given, ox->seed, (unsigned long long)step)))
                        return st;
                    if (n_inserted) *n_inserted += 2 * ox->n_o2;
                }
                if ((st = cell_sort(c))) return st;
            }
            simox_ctip_report rep;
            if ((st = ctip_solve(c, 0, &rep))) return st;
            simox_md_opts o2 = *o;
            // the rest of the step: FORCE, PME, VV2 (VV1 and CELL_SORT done)
            if ((st = ensure_gathered(c))) return st;
            if ((st = pme_fork(c, estep))) return st;
            if ((st = ensure_list(c))) return st;
            if ((st = eam_density(c, estep))) return st;
            if ((st = pair_forces(c, estep, want_rdf))) return st;
            cudaStreamWaitEvent(c->stream, c->ev_join, 0);
            if (stoch) st = nvt2_stoch(c, o2.dt, o2.alpha, o2.T_given, o2.seed, c->md_step_no, true, c->f_rec);
            else if (o2.thermostat) st = nvt2_berend(c, o2.dt, o2.T_given, true, c->f_rec);
            else st = vv2(c, o2.dt, true, c->f_rec);
            if (st) return st;
            continue;
        }
        // a graph replays only the launches it captured: the first step after
        // a new atom set (skin list seeded from the host) runs eagerly
        // stochastic steps stay eager too: their draws depend on the step number
        const bool graph_ok = c->graphs_on && !c->profiling && (!c->skin_mode || c->skin_valid) &&
                              !(o->thermostat && o->thermo_stoch);
        st = graph_ok ? md_step_graph(c, o, sort, estep, want_rdf) : md_step(c, o, sort, estep, want_rdf);
        if (st) return st;
    }
    if ((st = read_status(c))) return st;
    if (e) {
        cudaMemcpyAsync(c->h_acc, c->acc, sizeof(double) * A_COUNT, cudaMemcpyDeviceToHost, c->stream);
        if ((st = cuda_status(cudaStreamSynchronize(c->stream)))) return st;
        const double V = c->box[0] * c->box[1] * c->box[2];
        e->Epair = c->h_acc[A_EPAIR];
        e->Edir = c->h_acc[A_EDIR] * SX_KC;
        e->Ectip = c->h_acc[A_ECTIP] * SX_KC;
        e->Egroup = c->h_acc[A_EGROUP];
        e->Erec = SX_KC * c->h_acc[A_EREC] / V / SX_PI / 2.0;
        e->mv2 = c->h_acc[A_MV2];
        e->Eself = c->eself;
    }
    if (rdf) {
        std::vector<int> h(SIMOX_RDF_LEN);
        cudaMemcpyAsync(h.data(), c->rdf, sizeof(int) * SIMOX_RDF_LEN, cudaMemcpyDeviceToHost, c->stream);
        if ((st = cuda_status(cudaStreamSynchronize(c->stream)))) return st;
        for (int k = 0; k < SIMOX_RDF_LEN; k++) rdf[k] += h[k];
    }
    return SIMOX_OK;
}

}  // namespace sx

using namespace sx;

// POTENTIAL_SETUP datafmt.f90:142-262
extern "C" int simox_default_potential(simox_potential* P) {
    if (!P) return SIMOX_E_ARG;
    std::memset(P, 0, sizeof(*P));
    simox_metl* e = P->eam;
    const double tab[3][22] = {
        // r_e f_e rho_e rho_s alpha beta A B kappa lambda Fn(4) Fm(4) Fp(4)... split below
        {2.86392, 1.20378, 17.51747, 19.90041, 6.61317, 3.52702, 0.31487, 0.36555, 0.37985, 0.75969,
         -2.80760, -0.30144, 1.25856, -1.24760, -2.83000, 0.0, 0.62225, -2.48824, -2.83000, 0.0, 0.62225, -2.48824},
        {2.48875, 2.21149, 30.37003, 30.37137, 8.38345, 4.47117, 0.42905, 0.63353, 0.44360, 0.82066,
         -2.69351, -0.07644, 0.24144, -2.37563, -2.70000, 0.0, 0.26539, -0.15286, -2.70000, 0.0, 0.26539, 4.58568},
        {2.48199, 2.31453, 24.59573, 24.59573, 9.81827, 5.23641, 0.39281, 0.64624, 0.17031, 0.34061,
         -2.53499, -0.05960, 0.19306, -2.28232, -2.54000, 0.0, 0.20027, -0.14877, -2.54000, 0.0, 0.20027, 6.69465}};
    const double eta[3] = {0.78591, 1.01318, 1.18290}, Fe[3] = {-2.82453, -2.70839, -2.55187};
    for (int s = 0; s < 3; s++) {
        const double* t = tab[s];
        e[s].r_e = t[0]; e[s].f_e = t[1]; e[s].rho_e = t[2]; e[s].rho_s = t[3]; e[s].alpha = t[4];
        e[s].beta = t[5]; e[s].A = t[6]; e[s].B = t[7]; e[s].kappa = t[8]; e[s].lambda = t[9];
        for (int k = 0; k < 4; k++) { e[s].Fn[k] = t[10 + k]; e[s].Fm[k] = t[14 + k]; e[s].Fp[k] = t[18 + k]; }
        e[s].eta = eta[s]; e[s].Fe = Fe[s];
    }
    const double xm[5] = {26.981539, 58.6934, 55.84500, 15.9994, 1.00794};
    const double qmin[5] = {0.0, 0.0, 0.0, -2.0, 0.0}, qmax[5] = {3.0, 2.0, 3.0, 0.0, 0.0};
    const double chi[5] = {-1.47914, -1.70804, -1.90587, 2.000, 0.0};
    const double J[5] = {9.07222, 9.10954, 8.99819, 14.99523, 0.0};
    const double xi[5] = {0.968, 1.087, 1.024, 2.144, 0.0};
    const double Z[5] = {1.07514, 1.44450, 1.28612, 0.00, 0.0};
    for (int s = 0; s < 5; s++) {
        simox_potn& p = P->param[s];
        p.xm = xm[s]; p.qmin = qmin[s]; p.qmax = qmax[s]; p.chi = chi[s]; p.J = J[s]; p.xi = xi[s]; p.Z = Z[s];
    }
    // Slater 1s Coulomb-integral coefficients (datafmt.f90:201-220)
    for (int i = 0; i < 5; i++)
        for (int j = 0; j < 5; j++) sx::slater_fafb<double>(xi[i], xi[j], i == j, P->param[i].fafb[j]);
    simox_oxid& o = P->oxygn;
    const double ore[5] = {2.98520, 2.95732, 3.07992, 3.64857, 1.0};
    const double oal[5] = {8.49741, 7.96528, 7.52309, 5.44072, 0.0};
    const double obe[5] = {4.52114, 4.42411, 4.13330, 3.59746, 0.0};
    const double oA[5] = {0.09738, 0.13521, 0.17108, 0.34900, 0.0};
    const double oB[5] = {0.38121, 0.25332, 0.39869, 0.57438, 0.0};
    const double oka[5] = {0.18967, 0.47077, 0.22335, 0.08007, 0.0};
    const double ola[5] = {0.95234, 0.65524, 0.34380, 0.39310, 0.0};
    for (int s = 0; s < 5; s++) {
        o.r_e[s] = ore[s]; o.alph[s] = oal[s]; o.beta[s] = obe[s]; o.A[s] = oA[s]; o.B[s] = oB[s];
        o.kapp[s] = oka[s]; o.lamb[s] = ola[s];
    }
    const double F[5][4] = {{-1.56489, -1.39123, 1.77199, 1.59833},
                            {-1.58967, 1.30636, 9.81033, 0.0},
                            {-1.54116, 2.02821, 6.56240, 0.0},
                            {-1.51798, 2.30979, 7.69582, 0.0},
                            {-1.19082, 4.12936, 10.32338, 0.0}};
    for (int k = 0; k < 4; k++) {
        o.F0[k] = F[0][k]; o.F1[k] = F[1][k]; o.F2[k] = F[2][k]; o.F3[k] = F[3][k]; o.F4[k] = F[4][k];
    }
    const double re[5] = {54.62910, 64.26953, 66.21202, 66.92391, 74.23105};
    const double rmax[5] = {54.62910, 65.24078, 66.56797, 70.57748, 99.99999e9};
    for (int b = 0; b < 5; b++) { o.re[b] = re[b]; o.rmax[b] = rmax[b]; }
    o.fe = 1.39478; o.gamm = 2.11725; o.nu = 0.37457;
    return SIMOX_OK;
}

extern "C" const char* simox_status_string(int s) {
    switch (s) {
        case SIMOX_OK: return "ok";
        case SIMOX_E_ARG: return "bad argument";
        case SIMOX_E_CUDA: return "CUDA or cuFFT failure";
        case SIMOX_E_NOMEM: return "device allocation failed";
        case SIMOX_E_CELL_OVERFLOW: return "=== Cell particle limit crashed !!! ===";
        case SIMOX_E_NBR_OVERFLOW: return "=== neighbor particle limit crashed !!! === ";
        case SIMOX_E_UNKNOWN_PAIR: return "=== Unknown particle pair ===";
        case SIMOX_E_UNKNOWN_ELEMENT: return "# Unknown element";
        case SIMOX_E_BRENT: return "# **** Brent solver limit breached *** ";
        case SIMOX_E_CELL_TOO_SMALL: return "==== Error - unitcell is too small or cut-off radius is too small";
        case SIMOX_E_CAPACITY: return "more atoms than the context capacity";
        case SIMOX_E_POSITION: return "coordinate not finite or far outside the box";
        case SIMOX_E_CG_LIMIT: return "CG iteration cap reached";
        case SIMOX_E_FFT_SIZE: return "PME grid size not usable";
        case SIMOX_E_STATE: return "call order violated";
        case SIMOX_E_NO_DEVICE: return "no CUDA device";
        case SIMOX_E_UNSUPPORTED: return "hetero-metal pair form not implemented on the GPU path";
        case SIMOX_E_SCRATCH_LIMIT: return "size beyond the fixed scratch of simox_cell_sort_noalloc (65536 cells, stride 4096)";
        case SIMOX_E_IO: return "=== cannot open checkpoint, or not a checkpoint of this box ===";
        case SIMOX_E_RNG: return "random-force draw rejected 100 polar-method attempts";
        case SIMOX_E_SYNC: return "a device-wide wait inside a kernel gave up (its CTAs did not all arrive)";
        default: return "unknown status";
    }
}

extern "C" const char* simox_version(void) {
    return "simox_b200 1.0 (sm_100a; FP64 and mixed FP32/FP64 force, PME, CTIP, Verlet)";
}

static void free_ctx(simox_ctx* c) {
    if (!c) return;
    prof_collect(c);
    drop_graphs(c);
    adjoint_free(c);
    pme_free(c);
    void* bufs[] = {c->id, c->x, c->v, c->f, c->q, c->xm, c->cell_of, c->cell_xyz, c->cell_count, c->cell_start, c->cell_fill,
                    c->sorted, c->pair13, c->entries, c->xq_s, c->t_s, c->rec_s, c->frec_s, c->xo_s, c->nn, c->nbr, c->nn_max, c->nn_tot,
                    c->cs_count, c->cs_start, c->cs_fill, c->cs_cell_of, c->cs_entries, c->perm, c->x0,
                    c->skin_flag, c->nn_s, c->nbr_s, c->rho_s, c->dF_s, c->dF_f, c->tab_d, c->tab_f, c->c_const, c->g, c->pv, c->Ap, c->qs, c->jp,
                    c->act, c->line, c->acc, c->status, c->rdf, c->f_rec, c->rho_fx, c->fx_acc};
    for (void* p : bufs)
        if (p) cudaFree(p);
    if (c->h_acc) cudaFreeHost(c->h_acc);
    if (c->h_status) cudaFreeHost(c->h_status);
    for (auto ev : c->ev_pool) cudaEventDestroy(ev);
    for (auto& p : c->ev_pending) { cudaEventDestroy(p.second.first); cudaEventDestroy(p.second.second); }
    if (c->t0) cudaEventDestroy(c->t0);
    if (c->t1) cudaEventDestroy(c->t1);
    if (c->ev_fork) cudaEventDestroy(c->ev_fork);
    if (c->ev_join) cudaEventDestroy(c->ev_join);
    if (c->side) cudaStreamDestroy(c->side);
    if (c->stream) cudaStreamDestroy(c->stream);
    delete c;
}

template <typename T>
static bool dalloc(T** p, size_t count) {
    if (count == 0) count = 1;
    return cudaMalloc((void**)p, count * sizeof(T)) == cudaSuccess;
}

extern "C" int simox_create(const simox_setup* s, const simox_potential* pot, simox_ctx** out) {
    if (!s || !out) return SIMOX_E_ARG;
    *out = nullptr;
    if (s->n_atoms < 0 || s->rcut <= 0.0 || s->box[0] <= 0 || s->box[1] <= 0 || s->box[2] <= 0) return SIMOX_E_ARG;
    if (s->precision != SIMOX_FP64 && s->precision != SIMOX_MIXED) return SIMOX_E_ARG;
    const int order = s->pme_order ? s->pme_order : 4;
    if (order != 4 && order != 6 && order != 8) return SIMOX_E_ARG;
    for (int d = 0; d < 3; d++)
        if (s->fft[d] < order || s->fft[d] > 4096) return SIMOX_E_FFT_SIZE;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) return SIMOX_E_NO_DEVICE;
    if (s->device < 0 || s->device >= ndev) return SIMOX_E_ARG;
    if (cudaSetDevice(s->device) != cudaSuccess) return SIMOX_E_CUDA;

    simox_ctx* c = new (std::nothrow) simox_ctx();
    if (!c) return SIMOX_E_NOMEM;
    c->device = s->device;
    c->setup = *s;
    if (pot) c->pot = *pot;
    else simox_default_potential(&c->pot);
    c->n = s->n_atoms;
    c->cap = std::max(s->capacity, s->n_atoms);
    if ((size_t)c->cap > (size_t)sx::kIdxMask) {   // list entries hold 26-bit atom indices
        delete c;
        return SIMOX_E_CAPACITY;
    }
    c->precision = s->precision;
    c->flags = s->flags;
    c->order = order;
    c->npt_max = s->npt_max > 0 ? s->npt_max : SIMOX_NPT_MAX;
    c->nnb_cap = (c->flags & SIMOX_FLAG_REFERENCE_LIMITS) ? SIMOX_NNB_MAX : (s->nnb_max > 0 ? s->nnb_max : 1024);
    c->cap_s = 2 * c->nnb_cap;
    c->npt_max_s = std::max(2 * c->npt_max, 1024);
    c->skin = s->skin == 0.0 ? 1.0 : s->skin;
    for (int d = 0; d < 3; d++) {
        c->box[d] = s->box[d];
        c->inv_box[d] = 1.0 / s->box[d];
        c->hbox[d] = 0.5 * s->box[d];
        c->fft[d] = s->fft[d];
    }
    c->rcut = s->rcut;
    c->rcut2 = s->rcut * s->rcut;               // sys%Rcut**2 main.f90:253
    c->a = 3.8 / s->rcut;                        // main.f90:254 / force.f90:481
    c->dr_rdf = s->rcut / (double)SIMOX_NRDF;   // main.f90:334
    // cell grid main.f90:269-274
    for (int d = 0; d < 3; d++) {
        c->nc[d] = (int)(c->box[d] / c->rcut);
        c->lc[d] = c->box[d] / (double)c->nc[d];
    }
    if ((c->nc[0] < 3 && c->nc[1] < 3 && c->nc[2] < 3) || c->nc[0] < 2 || c->nc[1] < 2 || c->nc[2] < 2 ||
        c->nc[0] > 1024 || c->nc[1] > 1024 || c->nc[2] > 1024) {
        delete c;
        return SIMOX_E_CELL_TOO_SMALL;
    }
    // the FP32 staged-offset list build needs, per axis, Ncell >= 3 and
    // L/2 > Rcut + Lcell/2 (so a home atom's offset difference is the minimum image)
    c->fast_cells = true;
    for (int d = 0; d < 3; d++)
        if (c->nc[d] < 3 || !(0.5 * c->box[d] - c->rcut - 0.5 * c->lc[d] > 0.01)) c->fast_cells = false;
    c->ncell = c->nc[0] * c->nc[1] * c->nc[2];

    int st = SIMOX_OK;
    if (cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking) != cudaSuccess ||
        cudaStreamCreateWithFlags(&c->side, cudaStreamNonBlocking) != cudaSuccess ||
        cudaEventCreateWithFlags(&c->ev_fork, cudaEventDisableTiming) != cudaSuccess ||
        cudaEventCreateWithFlags(&c->ev_join, cudaEventDisableTiming) != cudaSuccess) {
        free_ctx(c);
        return SIMOX_E_CUDA;
    }
    const size_t N = (size_t)c->cap;
    bool ok = dalloc(&c->id, N) && dalloc(&c->x, 3 * N) && dalloc(&c->v, 3 * N) && dalloc(&c->f, 3 * N) && dalloc(&c->f_rec, 3 * N) &&
              dalloc(&c->q, N) && dalloc(&c->cell_of, N) && dalloc(&c->cell_xyz, N) && dalloc(&c->cell_count, c->ncell) &&
              dalloc(&c->cell_start, c->ncell + 1) && dalloc(&c->cell_fill, c->ncell) && dalloc(&c->sorted, N) &&
              dalloc(&c->pair13, (size_t)c->ncell * 13) && dalloc(&c->entries, (size_t)c->ncell * kEntries) &&
              dalloc(&c->xq_s, N) && dalloc(&c->t_s, N) && dalloc(&c->rec_s, N) && dalloc(&c->frec_s, N) &&
              dalloc(&c->xo_s, N) && dalloc(&c->nn, 2 * N) &&
              dalloc(&c->nbr, N * (size_t)c->nnb_cap) && dalloc(&c->nn_max, 1) && dalloc(&c->nn_tot, 1) &&
              dalloc(&c->rho_s, N) && dalloc(&c->dF_s, N) && dalloc(&c->dF_f, N) && dalloc(&c->rho_fx, N) &&
              dalloc(&c->fx_acc, 3 * N) && dalloc(&c->tab_d, kSpecies * kSpecies) &&
              dalloc(&c->tab_f, kSpecies * kSpecies) && dalloc(&c->line, 64) && dalloc(&c->acc, A_COUNT) &&
              dalloc(&c->status, 1) && dalloc(&c->rdf, SIMOX_RDF_LEN);
    if (!ok) { free_ctx(c); return SIMOX_E_NOMEM; }
    if (cudaMallocHost((void**)&c->h_acc, sizeof(double) * A_COUNT) != cudaSuccess ||
        cudaMallocHost((void**)&c->h_status, sizeof(int)) != cudaSuccess) {
        free_ctx(c);
        return SIMOX_E_NOMEM;
    }
    cudaMemsetAsync(c->acc, 0, sizeof(double) * A_COUNT, c->stream);
    cudaMemsetAsync(c->status, 0, sizeof(int), c->stream);
    cudaMemsetAsync(c->f, 0, sizeof(double) * 3 * N, c->stream);
    cudaMemsetAsync(c->v, 0, sizeof(double) * 3 * N, c->stream);
    cudaMemsetAsync(c->q, 0, sizeof(double) * N, c->stream);
    cudaEventCreate(&c->t0);
    cudaEventCreate(&c->t1);
    c->pair_order = c->sorted;
    if ((st = build_cell_tables(c)) || (st = setup_skin(c)) || (st = build_pair_tables(c)) || (st = pme_setup(c)) ||
        (st = ctip_alloc(c))) {
        free_ctx(c);
        return st;
    }
    *out = c;
    return cuda_status(cudaStreamSynchronize(c->stream));
}

extern "C" int simox_destroy(simox_ctx* c) {
    if (!c) return SIMOX_E_ARG;
    cudaSetDevice(c->device);
    cudaStreamSynchronize(c->stream);
    free_ctx(c);
    return SIMOX_OK;
}

extern "C" int simox_set_state(simox_ctx* c, int n, const int* id, const double* x, const double* v,
                               const double* f, const double* q) {
    if (!c || n < 0) return SIMOX_E_ARG;
    if (n > c->cap) return SIMOX_E_CAPACITY;
    if (!id && (!c->have_ids || n != c->n)) return SIMOX_E_ARG;
    cudaSetDevice(c->device);
    cudaStream_t s = c->stream;
    if (id) {
        bool has_h = false;
        int g0 = -1;   // species of the non-oxygen atoms: one (>= 0), several (-2) or none (-1)
        for (int i = 0; i < n; i++) {
            if (id[i] < 1 || id[i] > SIMOX_NATOM) return SIMOX_E_ARG;
            has_h |= id[i] == 5;
            if (id[i] != 4) g0 = (g0 == -1 || g0 == id[i] - 1) ? id[i] - 1 : -2;
        }
        c->has_h = has_h;
        c->g0_species = g0 >= 0 && g0 < 3 ? g0 : -1;
        cudaMemcpyAsync(c->id, id, sizeof(int) * n, cudaMemcpyHostToDevice, s);
        c->have_ids = true;
    }
    if (n != c->n) c->cells_valid = false;
    if (n != c->n || id) {
        c->skin_valid = false;
        drop_graphs(c);
    }
    c->n = n;
    if (x) cudaMemcpyAsync(c->x, x, sizeof(double) * 3 * n, cudaMemcpyHostToDevice, s);
    if (v) cudaMemcpyAsync(c->v, v, sizeof(double) * 3 * n, cudaMemcpyHostToDevice, s);
    if (f) cudaMemcpyAsync(c->f, f, sizeof(double) * 3 * n, cudaMemcpyHostToDevice, s);
    if (q) cudaMemcpyAsync(c->q, q, sizeof(double) * n, cudaMemcpyHostToDevice, s);
    if (x) {   // while the copies run: are all positions inside the box (no wrap needed)?
        const double hx = c->hbox[0], hy = c->hbox[1], hz = c->hbox[2];
        bool inb = true;
        for (int i = 0; i < n && inb; i++)
            inb = std::fabs(x[3 * i]) <= hx && std::fabs(x[3 * i + 1]) <= hy && std::fabs(x[3 * i + 2]) <= hz;
        c->in_box = inb;
        c->cells_fresh = false;
    }
    if (x || q || id) { c->gathered = false; c->list_valid = false; c->eam_valid = false; }
    return cuda_status(cudaStreamSynchronize(s));
}

extern "C" int simox_get_state(simox_ctx* c, int n, int* id, double* x, double* v, double* f, double* q) {
    if (!c || n != c->n) return SIMOX_E_ARG;
    cudaSetDevice(c->device);
    cudaStream_t s = c->stream;
    if (id) cudaMemcpyAsync(id, c->id, sizeof(int) * n, cudaMemcpyDeviceToHost, s);
    if (x) cudaMemcpyAsync(x, c->x, sizeof(double) * 3 * n, cudaMemcpyDeviceToHost, s);
    if (v) cudaMemcpyAsync(v, c->v, sizeof(double) * 3 * n, cudaMemcpyDeviceToHost, s);
    if (f) cudaMemcpyAsync(f, c->f, sizeof(double) * 3 * n, cudaMemcpyDeviceToHost, s);
    if (q) cudaMemcpyAsync(q, c->q, sizeof(double) * n, cudaMemcpyDeviceToHost, s);
    return cuda_status(cudaStreamSynchronize(s));
}

extern "C" int simox_get_natoms(simox_ctx* c, int* n) {
    if (!c || !n) return SIMOX_E_ARG;
    *n = c->n;
    return SIMOX_OK;
}

extern "C" int simox_cell_hierarchy(simox_ctx* c, int* ncell_out, int* pair) {
    if (!c) return SIMOX_E_ARG;
    if (ncell_out) for (int d = 0; d < 3; d++) ncell_out[d] = c->nc[d];
    if (pair) std::memcpy(pair, c->h_pair13.data(), c->h_pair13.size() * sizeof(int));
    return SIMOX_OK;
}

extern "C" int simox_cell_sort(simox_ctx* c) {
    if (!c) return SIMOX_E_ARG;
    cudaSetDevice(c->device);
    int st = sx::cell_sort(c);
    if (st) return st;
    st = read_status(c);
    if (st) c->cells_valid = false;
    return st;
}

extern "C" int simox_get_cells(simox_ctx* c, int* npt, int* link, int link_stride) {
    if (!c || !npt || !c->cells_valid) return c ? SIMOX_E_STATE : SIMOX_E_ARG;
    cudaSetDevice(c->device);
    if (int e = ensure_cell_lists(c)) return e;
    std::vector<int> start(c->ncell + 1), srt(std::max(c->n, 1));
    cudaMemcpyAsync(start.data(), c->cell_start, sizeof(int) * (c->ncell + 1), cudaMemcpyDeviceToHost, c->stream);
    cudaMemcpyAsync(srt.data(), c->sorted, sizeof(int) * c->n, cudaMemcpyDeviceToHost, c->stream);
    int st = cuda_status(cudaStreamSynchronize(c->stream));
    if (st) return st;
    for (int cc = 0; cc < c->ncell; cc++) {
        int m = start[cc + 1] - start[cc];
        npt[cc] = m;
        if (link) {
            if (m > link_stride) return SIMOX_E_CELL_OVERFLOW;
            for (int k = 0; k < m; k++) link[(size_t)cc * link_stride + k] = srt[start[cc] + k] + 1;
        }
    }
    return SIMOX_OK;
}

extern "C" int simox_pme_self(simox_ctx* c, simox_energies* e) {
    if (!c) return SIMOX_E_ARG;
    cudaSetDevice(c->device);
    cudaMemsetAsync(c->acc + A_Q2SUM, 0, 2 * sizeof(double), c->stream);
    int st = sx::pme_self(c);
    if (st) return st;
    cudaMemcpyAsync(c->h_acc, c->acc, sizeof(double) * A_COUNT, cudaMemcpyDeviceToHost, c->stream);
    if ((st = cuda_status(cudaStreamSynchronize(c->stream)))) return st;
    c->eself = c->h_acc[A_Q2SUM] * c->a / SX_SQRTPI * SX_KC + c->h_acc[A_ESUM];  // force.f90:498
    if (e) e->Eself = c->eself;
    return SIMOX_OK;
}

extern "C" int simox_get_psi(simox_ctx* c, double* psi) {
    if (!c || !psi) return SIMOX_E_ARG;
    if (!c->psi_valid) return SIMOX_E_STATE;
    cudaSetDevice(c->device);
    cudaMemcpyAsync(psi, c->psi, sizeof(double) * c->ngrid, cudaMemcpyDeviceToHost, c->stream);
    return cuda_status(cudaStreamSynchronize(c->stream));
}

extern "C" int simox_ctip_solve(simox_ctx* c, int max_cg, simox_energies* e, simox_ctip_report* rep) {
    if (!c) return SIMOX_E_ARG;
    cudaSetDevice(c->device);
    simox_ctip_report r{};
    int st = sx::ctip_solve(c, max_cg, &r);
    if (rep) *rep = r;
    if (st && st != SIMOX_E_CG_LIMIT) return st;
    if (e) e->Eself = c->eself;
    return st;
}

extern "C" int simox_force(simox_ctx* c, simox_energies* e, int* rdf) {
    if (!c) return SIMOX_E_ARG;
    cudaSetDevice(c->device);
    if (!c->cells_valid) return SIMOX_E_STATE;
    const bool eflag = e != nullptr;
    cudaMemsetAsync(c->acc, 0, sizeof(double) * (A_EGROUP + 1), c->stream);
    if (rdf) cudaMemsetAsync(c->rdf, 0, sizeof(int) * SIMOX_RDF_LEN, c->stream);
    int st;
    if ((st = ensure_list(c)) || (st = eam_density(c, eflag)) || (st = pair_forces(c, eflag, rdf != nullptr))) return st;
    if ((st = read_status(c))) return st;
    cudaMemcpyAsync(c->h_acc, c->acc, sizeof(double) * A_COUNT, cudaMemcpyDeviceToHost, c->stream);
    std::vector<int> h;
    if (rdf) {
        h.resize(SIMOX_RDF_LEN);
        cudaMemcpyAsync(h.data(), c->rdf, sizeof(int) * SIMOX_RDF_LEN, cudaMemcpyDeviceToHost, c->stream);
    }
    if ((st = cuda_status(cudaStreamSynchronize(c->stream)))) return st;
    if (rdf)
        for (int k = 0; k < SIMOX_RDF_LEN; k++) rdf[k] += h[k];
    if (e) {
        e->Epair = c->h_acc[A_EPAIR];
        e->Edir = c->h_acc[A_EDIR] * SX_KC;     // force.f90:251
        e->Ectip = c->h_acc[A_ECTIP] * SX_KC;   // force.f90:252
        e->Egroup = c->h_acc[A_EGROUP];
    }
    return SIMOX_OK;
}

extern "C" int simox_pme(simox_ctx* c, simox_energies* e) {
    if (!c) return SIMOX_E_ARG;
    cudaSetDevice(c->device);
    if (!c->cells_valid) return SIMOX_E_STATE;
    cudaMemsetAsync(c->acc + A_EREC, 0, sizeof(double), c->stream);
    int st = pme_forces(c, true, e != nullptr);
    if (st) return st;
    cudaMemcpyAsync(c->h_acc, c->acc, sizeof(double) * A_COUNT, cudaMemcpyDeviceToHost, c->stream);
    if ((st = cuda_status(cudaStreamSynchronize(c->stream)))) return st;
    if (e) {
        const double V = c->box[0] * c->box[1] * c->box[2];
        e->Erec = SX_KC * c->h_acc[A_EREC] / V / SX_PI / 2.0;  // force.f90:461
    }
    return SIMOX_OK;
}

extern "C" int simox_get_eam(simox_ctx* c, double* rho, double* dFdrho) {
    if (!c) return SIMOX_E_ARG;
    if (!c->eam_valid) return SIMOX_E_STATE;
    cudaSetDevice(c->device);
    const int n = c->n;
    std::vector<double> r(std::max(n, 1)), d(std::max(n, 1));
    std::vector<int> srt(std::max(n, 1));
    cudaMemcpyAsync(r.data(), c->rho_s, sizeof(double) * n, cudaMemcpyDeviceToHost, c->stream);
    cudaMemcpyAsync(d.data(), c->dF_s, sizeof(double) * n, cudaMemcpyDeviceToHost, c->stream);
    cudaMemcpyAsync(srt.data(), c->pair_order, sizeof(int) * n, cudaMemcpyDeviceToHost, c->stream);
    int st = cuda_status(cudaStreamSynchronize(c->stream));
    if (st) return st;
    for (int k = 0; k < n; k++) {
        if (rho) rho[srt[k]] = r[k];
        if (dFdrho) dFdrho[srt[k]] = d[k];
    }
    return SIMOX_OK;
}

static int read_mv2(simox_ctx* c, double* mv2) {
    int st = read_status(c);
    if (st) return st;
    if (mv2) {
        cudaMemcpyAsync(c->h_acc, c->acc, sizeof(double) * A_COUNT, cudaMemcpyDeviceToHost, c->stream);
        if ((st = cuda_status(cudaStreamSynchronize(c->stream)))) return st;
        *mv2 = c->h_acc[A_MV2];
    }
    return SIMOX_OK;
}

extern "C" int simox_vv_nve1(simox_ctx* c, double dt) {
    if (!c) return SIMOX_E_ARG;
    cudaSetDevice(c->device);
    int st = vv1(c, dt, false);
    return st ? st : cuda_status(cudaStreamSynchronize(c->stream));
}

extern "C" int simox_vv_nve1_reflect(simox_ctx* c, double dt) {
    if (!c) return SIMOX_E_ARG;
    cudaSetDevice(c->device);
    int st = vv1(c, dt, true);
    return st ? st : cuda_status(cudaStreamSynchronize(c->stream));
}

extern "C" int simox_vv_nve2(simox_ctx* c, double dt, double* mv2) {
    if (!c) return SIMOX_E_ARG;
    cudaSetDevice(c->device);
    int st = vv2(c, dt, false);
    return st ? st : read_mv2(c, mv2);
}

extern "C" int simox_vv_nvt2_berend(simox_ctx* c, double dt, double T_given, double* mv2) {
    if (!c) return SIMOX_E_ARG;
    cudaSetDevice(c->device);
    int st = nvt2_berend(c, dt, T_given, false);
    return st ? st : read_mv2(c, mv2);
}

extern "C" int simox_vv_nvt1_stoch(simox_ctx* c, double dt, double alpha) {
    if (!c) return SIMOX_E_ARG;
    cudaSetDevice(c->device);
    int st = nvt1_stoch(c, dt, alpha);
    return st ? st : cuda_status(cudaStreamSynchronize(c->stream));
}

extern "C" int simox_vv_nvt2_stoch(simox_ctx* c, double dt, double alpha, double T_given, unsigned long long seed,
                                   unsigned long long step, double* mv2) {
    if (!c || !(dt != 0.0) || !(alpha >= 0.0) || !(T_given >= 0.0)) return SIMOX_E_ARG;
    cudaSetDevice(c->device);
    int st = nvt2_stoch(c, dt, alpha, T_given, seed, step, false, nullptr);
    return st ? st : read_mv2(c, mv2);
}

// ---- binary FP64 checkpoint ------------------------------------------------
static const char kCkMagic[8] = {'S', 'I', 'M', 'O', 'X', 'C', 'K', '1'};

extern "C" int simox_checkpoint_write(simox_ctx* c, const char* path, long long step) {
    if (!c || !path) return SIMOX_E_ARG;
    if (!c->have_ids) return SIMOX_E_STATE;
    const int n = c->n;
    const size_t m = (size_t)std::max(n, 1);
    std::vector<int> id(m);
    std::vector<double> x(3 * m), v(3 * m), f(3 * m), q(m);
    int st = simox_get_state(c, n, id.data(), x.data(), v.data(), f.data(), q.data());
    if (st) return st;
    FILE* fp = std::fopen(path, "wb");
    if (!fp) return SIMOX_E_IO;
    const int32_t version = 1, nn = n;
    const int64_t s64 = step;
    bool ok = std::fwrite(kCkMagic, 1, 8, fp) == 8 && std::fwrite(&version, 4, 1, fp) == 1 &&
              std::fwrite(&nn, 4, 1, fp) == 1 && std::fwrite(&s64, 8, 1, fp) == 1 &&
              std::fwrite(c->box, 8, 3, fp) == 3;
    if (n > 0) {
        ok = ok && std::fwrite(id.data(), 4, (size_t)n, fp) == (size_t)n &&
             std::fwrite(x.data(), 8, 3 * (size_t)n, fp) == 3 * (size_t)n &&
             std::fwrite(v.data(), 8, 3 * (size_t)n, fp) == 3 * (size_t)n &&
             std::fwrite(f.data(), 8, 3 * (size_t)n, fp) == 3 * (size_t)n &&
             std::fwrite(q.data(), 8, (size_t)n, fp) == (size_t)n;
    }
    ok = (std::fclose(fp) == 0) && ok;
    return ok ? SIMOX_OK : SIMOX_E_IO;
}

extern "C" int simox_checkpoint_read(simox_ctx* c, const char* path, long long* step) {
    if (!c || !path) return SIMOX_E_ARG;
    FILE* fp = std::fopen(path, "rb");
    if (!fp) return SIMOX_E_IO;
    char magic[8];
    int32_t version = 0, nn = -1;
    int64_t s64 = 0;
    double box[3];
    bool ok = std::fread(magic, 1, 8, fp) == 8 && std::memcmp(magic, kCkMagic, 8) == 0 &&
              std::fread(&version, 4, 1, fp) == 1 && version == 1 && std::fread(&nn, 4, 1, fp) == 1 && nn >= 0 &&
              std::fread(&s64, 8, 1, fp) == 1 && std::fread(box, 8, 3, fp) == 3;
    ok = ok && box[0] == c->box[0] && box[1] == c->box[1] && box[2] == c->box[2];
    if (ok && nn > c->cap) {
        std::fclose(fp);
        return SIMOX_E_CAPACITY;
    }
    const size_t n = ok ? (size_t)nn : 0, m = std::max<size_t>(n, 1);
    std::vector<int> id(m);
    std::vector<double> x(3 * m), v(3 * m), f(3 * m), q(m);
    if (ok && n > 0) {
        ok = std::fread(id.data(), 4, n, fp) == n && std::fread(x.data(), 8, 3 * n, fp) == 3 * n &&
             std::fread(v.data(), 8, 3 * n, fp) == 3 * n && std::fread(f.data(), 8, 3 * n, fp) == 3 * n &&
             std::fread(q.data(), 8, n, fp) == n;
    }
    std::fclose(fp);
    if (!ok) return SIMOX_E_IO;
    const int st = simox_set_state(c, (int)n, id.data(), x.data(), v.data(), f.data(), q.data());
    if (st) return st;
    if (step) *step = (long long)s64;
    return SIMOX_OK;
}

// PRINT_STAT util.f90:3-19, FORMAT (ES11.4, 1X, F6.1, 5(1X, ES11.4))
extern "C" int simox_format_status(const simox_energies* e, int n_atoms, int step, double dt, char* buf, int len) {
    if (!e || !buf || len < 80 || n_atoms <= 0) return SIMOX_E_ARG;
    const double kB = 8.617343e-5;                                      // datafmt.f90:27
    const double E_es = e->Eself + e->Edir + e->Erec + e->Ectip;
    const double E_eam = e->Epair + e->Egroup;
    const double E_total = E_es + E_eam + e->mv2 / 2.0;
    const double T = e->mv2 / (double)(n_atoms * 3) / kB;
    char tf[32];
    std::snprintf(tf, sizeof(tf), "%6.1f", T);
    if (std::strlen(tf) > 6 || !std::isfinite(T)) std::snprintf(tf, sizeof(tf), "******");   // F6.1 overflow
    std::snprintf(buf, (size_t)len, "%11.4E %s %11.4E %11.4E %11.4E %11.4E %11.4E", (double)step * SX_TFM * dt, tf,
                  E_total, E_es, E_eam, e->Epair, e->Egroup);
    return SIMOX_OK;
}

// VINIT vverlet.f90:2-71
extern "C" int simox_vinit(simox_ctx* c, unsigned long long seed, double T_given, double dt, simox_energies* e,
                           double* mv2) {
    if (!c || !(T_given >= 0.0)) return SIMOX_E_ARG;
    cudaSetDevice(c->device);
    if (!c->cells_valid || !c->psi_valid) return SIMOX_E_STATE;
    const int n = c->n;
    double mv2_v = 0.0;
    int st = vinit_velocities(c, seed, T_given);
    if (st || (st = read_mv2(c, &mv2_v))) return st;
    if (mv2) *mv2 = mv2_v;
    if (n == 0) return SIMOX_OK;
    // forces at x - dt v (VV_NVE1 with -dt and zero forces), then x and v
    // back (vverlet.f90:57-70); v is unchanged by the zero-force kick
    double* x0 = nullptr;
    if (cudaMalloc(&x0, sizeof(double) * 3 * n) != cudaSuccess) {
        cudaGetLastError();
        return SIMOX_E_NOMEM;
    }
    const bool in_box = c->in_box;
    cudaMemcpyAsync(x0, c->x, sizeof(double) * 3 * n, cudaMemcpyDeviceToDevice, c->stream);
    cudaMemsetAsync(c->f, 0, sizeof(double) * 3 * n, c->stream);
    simox_energies ef{}, ep{};
    st = vv1(c, -dt, false);
    if (!st) st = simox_force(c, e ? &ef : nullptr, nullptr);
    if (!st) st = simox_pme(c, e ? &ep : nullptr);
    cudaMemcpyAsync(c->x, x0, sizeof(double) * 3 * n, cudaMemcpyDeviceToDevice, c->stream);
    const cudaError_t se = cudaStreamSynchronize(c->stream);
    cudaFree(x0);
    c->gathered = false;
    c->list_valid = false;
    c->eam_valid = false;
    c->cells_fresh = false;
    c->in_box = in_box;
    if (st) return st;
    if (se != cudaSuccess) return cuda_status(se);
    if (e) {
        *e = ef;
        e->Erec = ep.Erec;
        e->Eself = c->eself;
        e->mv2 = mv2_v;
    }
    return SIMOX_OK;
}

extern "C" int simox_md_run(simox_ctx* c, const simox_md_opts* o, int first_step, int nsteps, simox_energies* e,
                            int* rdf) {
    if (!c || !o || nsteps < 0) return SIMOX_E_ARG;
    cudaSetDevice(c->device);
    return md_run(c, o, first_step, nsteps, e, rdf);
}

// main.f90:63-84: the oxidation-mode loop
extern "C" int simox_md_run_oxidation(simox_ctx* c, const simox_md_opts* o, const simox_oxidation* ox,
                                      int first_step, int nsteps, simox_energies* e, int* rdf, int* n_inserted) {
    if (!c || !o || !ox || nsteps < 0 || ox->n_o2 < 0) return SIMOX_E_ARG;
    if (o->thermo_stoch) return SIMOX_E_ARG;   // the oxidation loop has no stochastic thermostat (main.f90:65-79)
    cudaSetDevice(c->device);
    if (n_inserted) *n_inserted = 0;
    return md_run(c, o, first_step, nsteps, e, rdf, ox, n_inserted);
}

extern "C" int simox_set_tuning(simox_ctx* c, const simox_tuning* t) {
    if (!c || !t) return SIMOX_E_ARG;
    if (t->force_splits < 1 || t->force_splits > 16) return SIMOX_E_ARG;
    if (t->force_splits != c->force_splits) {
        c->force_splits = t->force_splits;
        drop_graphs(c);   // the captured launches carry the old grid
    }
    return SIMOX_OK;
}

extern "C" int simox_get_tuning(simox_ctx* c, simox_tuning* t) {
    if (!c || !t) return SIMOX_E_ARG;
    t->force_splits = c->force_splits;
    t->half_list = c->using_skin && c->skin_half ? 1 : 0;
    return SIMOX_OK;
}

extern "C" int simox_timer_begin(simox_ctx* c) {
    if (!c) return SIMOX_E_ARG;
    return cuda_status(cudaEventRecord(c->t0, c->stream));
}

extern "C" int simox_timer_end(simox_ctx* c, float* ms) {
    if (!c || !ms) return SIMOX_E_ARG;
    cudaEventRecord(c->t1, c->stream);
    int st = cuda_status(cudaEventSynchronize(c->t1));
    if (st) return st;
    return cuda_status(cudaEventElapsedTime(ms, c->t0, c->t1));
}

extern "C" int simox_profile_enable(simox_ctx* c, int on) {
    if (!c) return SIMOX_E_ARG;
    if (!on) prof_collect(c);
    c->profiling = on != 0;
    return SIMOX_OK;
}

extern "C" int simox_profile_read(simox_ctx* c, char* buf, int buflen, double* ms, long long* launches, int cap,
                                  int* count) {
    if (!c) return SIMOX_E_ARG;
    prof_collect(c);
    const int n = (int)c->prof.names.size();
    if (count) *count = n;
    std::string all;
    for (int k = 0; k < n; k++) {
        if (k < cap) {
            if (ms) ms[k] = c->prof.ms[k];
            if (launches) launches[k] = c->prof.launches[k];
        }
        all += c->prof.names[k];
        all += '\n';
    }
    if (buf && buflen > 0) {
        std::strncpy(buf, all.c_str(), (size_t)buflen - 1);
        buf[buflen - 1] = 0;
    }
    return SIMOX_OK;
}

extern "C" int simox_profile_reset(simox_ctx* c) {
    if (!c) return SIMOX_E_ARG;
    prof_collect(c);
    std::fill(c->prof.ms.begin(), c->prof.ms.end(), 0.0);
    std::fill(c->prof.launches.begin(), c->prof.launches.end(), 0LL);
    return SIMOX_OK;
}

extern "C" int simox_launch_count(simox_ctx* c, long long* n) {
    if (!c || !n) return SIMOX_E_ARG;
    *n = c->launches;
    return SIMOX_OK;
}

extern "C" int simox_sync(simox_ctx* c) {
    if (!c) return SIMOX_E_ARG;
    return cuda_status(cudaStreamSynchronize(c->stream));
}

extern "C" int simox_skin_rebuilds(simox_ctx* c, long long* n) {
    if (!c || !n) return SIMOX_E_ARG;
    int v[2] = {0, 0};
    if (c->skin_flag) cudaMemcpyAsync(v, c->skin_flag, sizeof(v), cudaMemcpyDeviceToHost, c->stream);
    int st = cuda_status(cudaStreamSynchronize(c->stream));
    *n = v[1];
    return st;
}

extern "C" int simox_neighbor_stats(simox_ctx* c, int* max_nnb, long long* total_nnb) {
    if (!c) return SIMOX_E_ARG;
    int mx = 0;
    unsigned long long tot = 0;
    cudaMemcpyAsync(&mx, c->nn_max, sizeof(int), cudaMemcpyDeviceToHost, c->stream);
    cudaMemcpyAsync(&tot, c->nn_tot, sizeof(tot), cudaMemcpyDeviceToHost, c->stream);
    int st = cuda_status(cudaStreamSynchronize(c->stream));
    if (max_nnb) *max_nnb = mx;
    if (total_nnb) *total_nnb = (long long)tot;
    return st;
}
