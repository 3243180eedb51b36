// batch.cu -- many independent systems advanced together (no counterpart in
// the reference, which runs one system per process).
//
// Each system is an ordinary context.  One MD step of every system
// (VV_NVE1, CELL_SORT, FORCE with PME on a side branch, VV2 / NVT) is
// captured into ONE CUDA graph: a master stream forks every context's stream,
// each records its step, and all join back.  Replaying that graph advances
// all systems with a single launch per step; the GPU runs the systems'
// kernels concurrently, so small systems share the SMs instead of each
// underfilling them in turn.
//
// The autotuner chooses the force pass's CTAs per skin cell for every system
// from one rule ("enough CTAs for `target` in total"), timing each candidate
// on the whole batch, because with concurrent systems the best split is a
// property of the batch, not of one system alone.
#include "simox_internal.cuh"

#include <algorithm>
#include <cmath>
#include <vector>

struct simox_batch {
    std::vector<simox_ctx*> ctx;
    int device = 0;
    cudaStream_t master = nullptr;
    cudaEvent_t fork = nullptr, t0 = nullptr, t1 = nullptr;
    std::vector<cudaEvent_t> join;
    struct G {
        unsigned key = 0;
        cudaGraphExec_t exec = nullptr;
        long long kernels = 0;
        // what the captured launches baked in: each member's step options
        // (dt, thermostat, T_given, reflect) and its graph generation (bumped
        // by tuning changes and new atom sets)
        std::vector<simox_md_opts> opts;
        std::vector<unsigned long long> gens;
    };
    G graphs[2];
    long long launches = 0;
    bool primed = false;       // every context has run one eager step
};

namespace {

void drop(simox_batch* b) {
    for (auto& g : b->graphs) {
        if (g.exec) cudaGraphExecDestroy(g.exec);
        g = simox_batch::G{};
    }
}

int check_opts(const simox_batch* b, const simox_md_opts* o) {
    for (size_t k = 0; k < b->ctx.size(); k++) {
        if (o[k].freq_new != 0 || o[k].charge_every_step) return SIMOX_E_ARG;
        if (o[k].freq_sort != o[0].freq_sort || o[k].freq_stat != o[0].freq_stat) return SIMOX_E_ARG;
        if (o[k].accumulate_rdf) return SIMOX_E_ARG;
        if (o[k].thermostat && o[k].thermo_stoch) return SIMOX_E_ARG;   // per-step draws: not graph-replayable
        if (!b->ctx[k]->psi_valid || !b->ctx[k]->cells_valid) return SIMOX_E_STATE;
    }
    return SIMOX_OK;
}

// one step of every system, each on its own stream (eager or under capture)
int step_all(simox_batch* b, const simox_md_opts* o, bool sort, bool estep) {
    cudaEventRecord(b->fork, b->master);
    for (size_t k = 0; k < b->ctx.size(); k++) {
        simox_ctx* c = b->ctx[k];
        cudaStreamWaitEvent(c->stream, b->fork, 0);
        if (int st = sx::md_step(c, &o[k], sort, estep, false)) return st;
        cudaEventRecord(b->join[k], c->stream);
        cudaStreamWaitEvent(b->master, b->join[k], 0);
    }
    return sx::cuda_status(cudaGetLastError());
}

// The options a captured step reads as kernel arguments.
bool same_step_opts(const simox_md_opts& a, const simox_md_opts& b) {
    return a.dt == b.dt && a.thermostat == b.thermostat && a.T_given == b.T_given && a.reflect == b.reflect;
}

bool graph_current(const simox_batch* b, const simox_batch::G& g, const simox_md_opts* o) {
    if (g.opts.size() != b->ctx.size() || g.gens.size() != b->ctx.size()) return false;
    for (size_t k = 0; k < b->ctx.size(); k++)
        if (g.gens[k] != b->ctx[k]->graph_gen || !same_step_opts(g.opts[k], o[k])) return false;
    return true;
}

int graph_step(simox_batch* b, const simox_md_opts* o, bool sort, bool estep) {
    const unsigned key = 1u | (sort ? 2u : 0u) | (estep ? 4u : 0u);
    simox_batch::G* hit = nullptr;
    for (auto& g : b->graphs)
        if (g.exec && g.key == key && graph_current(b, g, o)) hit = &g;
    if (!hit) {
        long long l0 = 0;
        for (auto* c : b->ctx) l0 += c->launches;
        if (cudaStreamBeginCapture(b->master, cudaStreamCaptureModeThreadLocal) != cudaSuccess) return SIMOX_E_CUDA;
        int st = step_all(b, o, sort, estep);
        cudaGraph_t graph = nullptr;
        const cudaError_t ce = cudaStreamEndCapture(b->master, &graph);
        cudaGetLastError();
        if (st || ce != cudaSuccess || !graph) {
            if (graph) cudaGraphDestroy(graph);
            return st ? st : SIMOX_E_CUDA;
        }
        cudaGraphExec_t exec = nullptr;
        const cudaError_t ie = cudaGraphInstantiate(&exec, graph, 0);
        cudaGraphDestroy(graph);
        if (ie != cudaSuccess) return SIMOX_E_CUDA;
        long long l1 = 0;
        for (auto* c : b->ctx) l1 += c->launches;
        simox_batch::G& g = b->graphs[estep ? 1 : 0];
        if (g.exec) cudaGraphExecDestroy(g.exec);
        g.key = key;
        g.exec = exec;
        g.kernels = l1 - l0;
        g.opts.assign(o, o + b->ctx.size());
        g.gens.clear();
        for (auto* c : b->ctx) g.gens.push_back(c->graph_gen);
        hit = &g;
    }
    b->launches += hit->kernels;
    return sx::cuda_status(cudaGraphLaunch(hit->exec, b->master));
}

int run(simox_batch* b, const simox_md_opts* o, int first, int nsteps) {
    for (int step = first; step < first + nsteps; step++) {
        const bool sort = o[0].freq_sort > 0 && step % o[0].freq_sort == 0;
        const bool estep = o[0].freq_stat <= 0 || step % o[0].freq_stat == 0;
        int st;
        // a member whose skin list must be seeded from the host (new atom set)
        // cannot be captured: that step runs eagerly, as in simox_md_run
        bool seed = false;
        for (auto* c : b->ctx) seed |= c->skin_mode && !c->skin_valid;
        if (!b->primed || seed) {
            // the first step after set-up seeds each skin list: eager
            long long l0 = 0, l1 = 0;
            for (auto* c : b->ctx) l0 += c->launches;
            st = step_all(b, o, sort, estep);
            for (auto* c : b->ctx) l1 += c->launches;
            b->launches += l1 - l0;
            b->primed = true;
        } else {
            st = graph_step(b, o, sort, estep);
        }
        if (st) return st;
    }
    return SIMOX_OK;
}

}  // namespace

extern "C" int simox_batch_create(int nsys, simox_ctx* const* ctxs, simox_batch** out) {
    if (!out || nsys <= 0 || !ctxs) return SIMOX_E_ARG;
    *out = nullptr;
    for (int k = 0; k < nsys; k++)
        if (!ctxs[k] || ctxs[k]->device != ctxs[0]->device) return SIMOX_E_ARG;
    simox_batch* b = new simox_batch;
    b->ctx.assign(ctxs, ctxs + nsys);
    b->device = ctxs[0]->device;
    cudaSetDevice(b->device);
    bool ok = cudaStreamCreateWithFlags(&b->master, cudaStreamNonBlocking) == cudaSuccess &&
              cudaEventCreateWithFlags(&b->fork, cudaEventDisableTiming) == cudaSuccess &&
              cudaEventCreate(&b->t0) == cudaSuccess && cudaEventCreate(&b->t1) == cudaSuccess;
    b->join.assign(nsys, nullptr);
    for (int k = 0; ok && k < nsys; k++) ok = cudaEventCreateWithFlags(&b->join[k], cudaEventDisableTiming) == cudaSuccess;
    if (!ok) {
        simox_batch_destroy(b);
        return SIMOX_E_CUDA;
    }
    *out = b;
    return SIMOX_OK;
}

extern "C" int simox_batch_destroy(simox_batch* b) {
    if (!b) return SIMOX_E_ARG;
    cudaSetDevice(b->device);
    if (b->master) cudaStreamSynchronize(b->master);
    drop(b);
    for (auto e : b->join)
        if (e) cudaEventDestroy(e);
    if (b->fork) cudaEventDestroy(b->fork);
    if (b->t0) cudaEventDestroy(b->t0);
    if (b->t1) cudaEventDestroy(b->t1);
    if (b->master) cudaStreamDestroy(b->master);
    delete b;
    return SIMOX_OK;
}

extern "C" int simox_batch_md_run(simox_batch* b, const simox_md_opts* opts, int first_step, int nsteps,
                                  simox_energies* last) {
    if (!b || !opts || nsteps < 0) return SIMOX_E_ARG;
    cudaSetDevice(b->device);
    int st = check_opts(b, opts);
    if (st) return st;
    // energies of the last energy step: zeroed by the step that evaluates them
    if ((st = run(b, opts, first_step, nsteps))) return st;
    if ((st = sx::cuda_status(cudaStreamSynchronize(b->master)))) return st;
    for (size_t k = 0; k < b->ctx.size(); k++) {
        simox_ctx* c = b->ctx[k];
        if ((st = sx::read_status(c))) return st;
        if (!last) continue;
        cudaMemcpyAsync(c->h_acc, c->acc, sizeof(double) * sx::A_COUNT, cudaMemcpyDeviceToHost, c->stream);
        if ((st = sx::cuda_status(cudaStreamSynchronize(c->stream)))) return st;
        const double V = c->box[0] * c->box[1] * c->box[2];
        simox_energies& e = last[k];
        e.Epair = c->h_acc[sx::A_EPAIR];
        e.Edir = c->h_acc[sx::A_EDIR] * SX_KC;
        e.Ectip = c->h_acc[sx::A_ECTIP] * SX_KC;
        e.Egroup = c->h_acc[sx::A_EGROUP];
        e.Erec = SX_KC * c->h_acc[sx::A_EREC] / V / SX_PI / 2.0;
        e.mv2 = c->h_acc[sx::A_MV2];
        e.Eself = c->eself;
    }
    return SIMOX_OK;
}

extern "C" int simox_batch_autotune(simox_batch* b, const simox_md_opts* opts, int first_step, int trial_steps,
                                    double* times_ms, int* best) {
    if (!b || !opts || trial_steps < 1) return SIMOX_E_ARG;
    cudaSetDevice(b->device);
    int st = check_opts(b, opts);
    if (st) return st;
    static const int targets[5] = {0, 148, 296, 592, 1184};
    double t[5];
    int step = first_step;
    for (int i = 0; i < 5; i++) {
        for (auto* c : b->ctx) {
            const int nc = std::max(1, c->ncell_s);
            const int s = targets[i] == 0 ? 1 : std::max(1, std::min(16, (targets[i] + nc - 1) / nc));
            if (s != c->force_splits) {
                c->force_splits = s;
                sx::drop_graphs(c);
            }
        }
        drop(b);
        if ((st = run(b, opts, step, 1))) return st;   // capture (untimed)
        step += 1;
        cudaEventRecord(b->t0, b->master);
        if ((st = run(b, opts, step, trial_steps))) return st;
        step += trial_steps;
        cudaEventRecord(b->t1, b->master);
        if ((st = sx::cuda_status(cudaEventSynchronize(b->t1)))) return st;
        float ms = 0.f;
        cudaEventElapsedTime(&ms, b->t0, b->t1);
        t[i] = ms / trial_steps;
    }
    int k = (int)(std::min_element(t, t + 5) - t);
    for (auto* c : b->ctx) {
        const int nc = std::max(1, c->ncell_s);
        const int s = targets[k] == 0 ? 1 : std::max(1, std::min(16, (targets[k] + nc - 1) / nc));
        if (s != c->force_splits) {
            c->force_splits = s;
            sx::drop_graphs(c);
        }
    }
    drop(b);
    if (times_ms)
        for (int i = 0; i < 5; i++) times_ms[i] = t[i];
    if (best) *best = k;
    for (auto* c : b->ctx)
        if ((st = sx::read_status(c))) return st;
    return SIMOX_OK;
}

extern "C" int simox_batch_launch_count(simox_batch* b, long long* n) {
    if (!b || !n) return SIMOX_E_ARG;
    *n = b->launches;
    return SIMOX_OK;
}
