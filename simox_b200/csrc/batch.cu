// batch.cu -- many independent systems advanced together (no counterpart in
// the reference, which runs one system per process).
//
// Each system is an ordinary context.  A batch step is built once per step
// kind (sort / energy step) and replayed as one CUDA graph:
//
// * per pass (the default): every member's MD step (VV_NVE1, CELL_SORT,
//   FORCE with PME on a side lane, VV2 / NVT) is recorded, not issued
//   (simox_batched.cuh); when all members recorded the same sequence, each
//   kernel of the sequence is launched ONCE for all systems over a work list
//   of (system, block) -- the batched instance of the kernel's body reads its
//   system's arguments from a device table -- the byte fills of a step
//   position become one fill launch, and the FFTs of systems with the same
//   grid run as one batched cuFFT plan.  A step of 256 systems is then about
//   30 launches instead of about 23 per system.
// * per system (the fallback when the sequences differ, or on request): a
//   master stream forks every context's stream, each records its ordinary
//   step, and all join back; the graph holds every system's own launches.
//
// The autotuner chooses the force pass's CTAs per skin cell for every system
// from one rule ("enough CTAs for `target` in total"), timing each candidate
// on the whole batch, because with concurrent systems the best split is a
// property of the batch, not of one system alone.
#include "simox_internal.cuh"

#include <algorithm>
#include <cmath>
#include <vector>

namespace {

// The batched plan of a group of members with the same grid and precision;
// its strided buffers stand in for the members' grids while they record.
struct FftGroup {
    bool dbl = false;
    int K[3] = {0, 0, 0};
    std::vector<int> members;
    size_t ngrid = 0, nhalf = 0;
    void* real = nullptr;     // members' real grids, ngrid apart
    void* cplx = nullptr;     // members' half spectra, nhalf apart
    cufftHandle r2c = 0, c2r = 0;
};

struct FftPool {
    std::vector<FftGroup> groups;
    ~FftPool() { release(); }
    void release() {
        for (auto& g : groups) {
            if (g.r2c) cufftDestroy(g.r2c);
            if (g.c2r) cufftDestroy(g.c2r);
            if (g.real) cudaFree(g.real);
            if (g.cplx) cudaFree(g.cplx);
        }
        groups.clear();
    }
};

}  // namespace

struct simox_batch {
    std::vector<simox_ctx*> ctx;
    int device = 0;
    cudaStream_t master = nullptr;
    cudaStream_t side = nullptr;            // the PME lane of a per-pass step
    cudaEvent_t fork = nullptr, t0 = nullptr, t1 = nullptr;
    cudaEvent_t lane_ev[2] = {nullptr, nullptr};   // per-pass step: fork and join of the PME lane
    std::vector<cudaEvent_t> join;
    struct G {
        unsigned key = 0;
        cudaGraphExec_t exec = nullptr;
        long long kernels = 0;
        int mode = SIMOX_BATCH_PER_SYSTEM;
        void* tables = nullptr;             // per pass: argument packs, work lists, fill items
        // what the captured launches baked in: each member's step options
        // (dt, thermostat, T_given, reflect) and its graph generation (bumped
        // by tuning changes and new atom sets)
        std::vector<simox_md_opts> opts;
        std::vector<unsigned long long> gens;
    };
    G graphs[2];
    FftPool pool;                           // batched FFT plans and their grids (kept across graphs)
    long long launches = 0;
    bool primed = false;       // every context has run one eager step
    int want_mode = SIMOX_BATCH_PER_PASS;
    int last_mode = SIMOX_BATCH_PER_SYSTEM;
    bool per_pass_failed = false;           // the members' steps could not be merged
    std::vector<unsigned long long> pool_gens;   // members' graph generations when the pool was made
};

namespace {

void drop(simox_batch* b) {
    bool busy = false;
    for (auto& g : b->graphs) busy |= g.exec != nullptr;
    if (busy) cudaStreamSynchronize(b->master);   // a replay in flight still reads the tables
    for (auto& g : b->graphs) {
        if (g.exec) cudaGraphExecDestroy(g.exec);
        if (g.tables) cudaFree(g.tables);
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

// ---------------------------------------------------------------------------
// per-pass steps

// the byte fills of one step position, one block per member range
__global__ void __launch_bounds__(256) batched_fill_kernel(const sx::FillItem* __restrict__ items) {
    const sx::FillItem it = items[blockIdx.x];
    unsigned char* p = static_cast<unsigned char*>(it.p);
    const unsigned char v = (unsigned char)it.value;
    const unsigned long long n = it.bytes;
    const unsigned long long mis = (16ull - ((unsigned long long)(uintptr_t)p & 15ull)) & 15ull;
    const unsigned long long head = mis < n ? mis : n;
    for (unsigned long long k = threadIdx.x; k < head; k += blockDim.x) p[k] = v;
    const unsigned long long nv = (n - head) / 16;
    uint4* q = reinterpret_cast<uint4*>(p + head);
    const unsigned w = 0x01010101u * v;
    for (unsigned long long k = threadIdx.x; k < nv; k += blockDim.x) q[k] = make_uint4(w, w, w, w);
    for (unsigned long long k = head + 16 * nv + threadIdx.x; k < n; k += blockDim.x) p[k] = v;
}

size_t align_up(size_t x, size_t a) { return (x + a - 1) / a * a; }

// every PME resource of every member joins the group of its grid
int make_fft_groups(simox_batch* b, FftPool& pool) {
    for (size_t k = 0; k < b->ctx.size(); k++) {
        simox_ctx* c = b->ctx[k];
        for (sx::PmeRes& R : c->pme) {
            if (!R.ready) continue;
            FftGroup* g = nullptr;
            for (auto& h : pool.groups)
                if (h.dbl == R.dbl && h.K[0] == c->fft[0] && h.K[1] == c->fft[1] && h.K[2] == c->fft[2]) g = &h;
            if (!g) {
                pool.groups.emplace_back();
                g = &pool.groups.back();
                g->dbl = R.dbl;
                for (int d = 0; d < 3; d++) g->K[d] = c->fft[d];
                g->ngrid = c->ngrid;
                g->nhalf = c->nhalf;
            }
            g->members.push_back((int)k);
        }
    }
    for (auto& g : pool.groups) {
        const size_t m = g.members.size();
        const size_t es = g.dbl ? sizeof(double) : sizeof(float);
        if (cudaMalloc(&g.real, m * g.ngrid * es) != cudaSuccess) return SIMOX_E_NOMEM;
        if (cudaMalloc(&g.cplx, m * g.nhalf * 2 * es) != cudaSuccess) return SIMOX_E_NOMEM;
        int n[3] = {g.K[2], g.K[1], g.K[0]};   // slowest first; x contiguous
        if (cufftPlanMany(&g.r2c, 3, n, nullptr, 1, (int)g.ngrid, nullptr, 1, (int)g.nhalf,
                          g.dbl ? CUFFT_D2Z : CUFFT_R2C, (int)m) != CUFFT_SUCCESS)
            return SIMOX_E_FFT_SIZE;
        if (cufftPlanMany(&g.c2r, 3, n, nullptr, 1, (int)g.nhalf, nullptr, 1, (int)g.ngrid,
                          g.dbl ? CUFFT_Z2D : CUFFT_C2R, (int)m) != CUFFT_SUCCESS)
            return SIMOX_E_FFT_SIZE;
    }
    return SIMOX_OK;
}

// Record one member's step.  Launches that bypass the recorder would run
// for real: both of the context's streams are held in throw-away captures,
// and a capture that caught anything marks the recording unusable.
int record_member(simox_ctx* c, const simox_md_opts* o, bool sort, bool estep, sx::Recorder& R) {
    R.main = c->stream;
    R.side = c->side;
    const bool cap1 = cudaStreamBeginCapture(c->stream, cudaStreamCaptureModeThreadLocal) == cudaSuccess;
    const bool cap2 = cudaStreamBeginCapture(c->side, cudaStreamCaptureModeThreadLocal) == cudaSuccess;
    c->rec = &R;
    const int st = sx::md_step(c, o, sort, estep, false);
    c->rec = nullptr;
    cudaGraph_t g1 = nullptr, g2 = nullptr;
    if (cap2) cudaStreamEndCapture(c->side, &g2);
    if (cap1) cudaStreamEndCapture(c->stream, &g1);
    cudaGetLastError();
    size_t n1 = 0, n2 = 0;
    if (g1) cudaGraphGetNodes(g1, nullptr, &n1);
    if (g2) cudaGraphGetNodes(g2, nullptr, &n2);
    if (g1) cudaGraphDestroy(g1);
    if (g2) cudaGraphDestroy(g2);
    if (!cap1 || !cap2 || n1 || n2) R.bad = true;
    return st;
}

bool same_op(const sx::RecOp& a, const sx::RecOp& b) {
    if (a.kind != b.kind || a.lane != b.lane) return false;
    switch (a.kind) {
        case sx::RecOp::KERNEL: return a.fn == b.fn && a.threads == b.threads && a.args.size() == b.args.size();
        case sx::RecOp::EV_RECORD:
        case sx::RecOp::EV_WAIT: return a.tag == b.tag;
        case sx::RecOp::FFT: return a.fft == b.fft;
        default: return true;
    }
}

// The group whose buffers a recorded FFT reads: the member's slot in it.
const FftGroup* fft_group_of(const FftPool& pool, const sx::RecOp& op, int k, int* slot) {
    for (const auto& g : pool.groups) {
        if (g.dbl != (op.fft >= 2)) continue;
        for (size_t j = 0; j < g.members.size(); j++) {
            if (g.members[j] != k) continue;
            const size_t es = g.dbl ? sizeof(double) : sizeof(float);
            const char* re = static_cast<const char*>(g.real) + j * g.ngrid * es;
            const char* cx = static_cast<const char*>(g.cplx) + j * g.nhalf * 2 * es;
            const bool fwd = op.fft == 0 || op.fft == 2;
            const void* src = fwd ? (const void*)re : (const void*)cx;
            const void* dst = fwd ? (const void*)cx : (const void*)re;
            if (op.in == src && op.out == dst) {
                *slot = (int)j;
                return &g;
            }
        }
    }
    return nullptr;
}

// Build the per-pass graph of one step kind.  Returns SIMOX_OK with
// g.exec set, SIMOX_OK with g.exec null when the members' steps cannot be
// merged (the caller falls back to the per-system graph), or an error.
int capture_per_pass(simox_batch* b, const simox_md_opts* o, bool sort, bool estep, FftPool& pool,
                     simox_batch::G& out) {
    const int nsys = (int)b->ctx.size();
    // without the batched plans' buffers (no memory for them, or a plan
    // cuFFT refuses) every member's FFTs run on its own plan
    if (pool.groups.empty() && make_fft_groups(b, pool) != SIMOX_OK) {
        pool.release();
        cudaGetLastError();
    }
    // record with the members' grids lent from the batched plans' buffers
    std::vector<sx::Recorder> rec(nsys);
    bool ok = true;
    for (int k = 0; k < nsys; k++) {
        simox_ctx* c = b->ctx[k];
        struct Lent { sx::PmeRes* R; void* grid; void* cgrid; };
        std::vector<Lent> lent;
        for (sx::PmeRes& R : c->pme) {
            if (!R.ready) continue;
            for (const auto& g : pool.groups) {
                if (g.dbl != R.dbl) continue;
                for (size_t j = 0; j < g.members.size(); j++)
                    if (g.members[j] == k && g.K[0] == c->fft[0] && g.K[1] == c->fft[1] && g.K[2] == c->fft[2]) {
                        const size_t es = g.dbl ? sizeof(double) : sizeof(float);
                        lent.push_back({&R, R.grid, R.cgrid});
                        R.grid = static_cast<char*>(g.real) + j * g.ngrid * es;
                        R.cgrid = static_cast<char*>(g.cplx) + j * g.nhalf * 2 * es;
                    }
            }
        }
        const int st = record_member(c, &o[k], sort, estep, rec[k]);
        for (auto& l : lent) {
            l.R->grid = l.grid;
            l.R->cgrid = l.cgrid;
        }
        sx::pme_bind_stream(c);
        if (st) return st;
        ok = ok && !rec[k].bad && rec[k].ops.size() == rec[0].ops.size();
    }
    const size_t nops = rec[0].ops.size();
    for (int k = 1; ok && k < nsys; k++)
        for (size_t i = 0; ok && i < nops; i++) ok = same_op(rec[0].ops[i], rec[k].ops[i]);
    if (!ok) return SIMOX_OK;

    // tables: per kernel position the members' argument packs and the block
    // prefix; per fill run the members' ranges
    struct Item { int kind; int lane; size_t pos; size_t off_a, off_b; unsigned blocks; size_t smem; int count; };
    std::vector<Item> items;
    std::vector<unsigned char> host;
    auto reserve = [&](size_t bytes, size_t al) {
        const size_t off = align_up(host.size(), al);
        host.resize(off + bytes);
        return off;
    };
    for (size_t i = 0; i < nops; i++) {
        const sx::RecOp& op0 = rec[0].ops[i];
        if (op0.kind == sx::RecOp::KERNEL) {
            const size_t psz = op0.args.size();
            const size_t oa = reserve(psz * nsys, 256);
            for (int k = 0; k < nsys; k++) std::memcpy(host.data() + oa + psz * k, rec[k].ops[i].args.data(), psz);
            const size_t ob = reserve(sizeof(int) * (nsys + 1), 16);
            int* bs = reinterpret_cast<int*>(host.data() + ob);
            long long tot = 0;
            size_t smem = 0;
            bs[0] = 0;
            for (int k = 0; k < nsys; k++) {
                tot += rec[k].ops[i].grid;
                smem = std::max(smem, rec[k].ops[i].smem);
                bs = reinterpret_cast<int*>(host.data() + ob);
                bs[k + 1] = (int)tot;
            }
            if (tot > 0x7fffffffLL) return SIMOX_E_ARG;
            items.push_back({sx::RecOp::KERNEL, op0.lane, i, oa, ob, (unsigned)tot, smem, 0});
        } else if (op0.kind == sx::RecOp::MEMSET) {
            // consecutive fills of a lane: one launch
            size_t j = i;
            while (j + 1 < nops && rec[0].ops[j + 1].kind == sx::RecOp::MEMSET && rec[0].ops[j + 1].lane == op0.lane)
                j++;
            std::vector<sx::FillItem> fills;
            bool one_value = true;
            for (size_t m = i; m <= j; m++)
                for (int k = 0; k < nsys; k++) {
                    const sx::RecOp& r = rec[k].ops[m];
                    one_value = one_value && r.value == op0.value;
                    if (r.bytes) fills.push_back({r.ptr, (unsigned long long)r.bytes, r.value, 0});
                }
            if (!one_value) {   // fills of different values may overlap: keep them in order
                j = i;
                fills.clear();
                for (int k = 0; k < nsys; k++) {
                    const sx::RecOp& r = rec[k].ops[i];
                    if (r.bytes) fills.push_back({r.ptr, (unsigned long long)r.bytes, r.value, 0});
                }
            }
            const size_t oa = reserve(sizeof(sx::FillItem) * fills.size(), 16);
            if (!fills.empty()) std::memcpy(host.data() + oa, fills.data(), sizeof(sx::FillItem) * fills.size());
            items.push_back({sx::RecOp::MEMSET, op0.lane, i, oa, 0, 0, 0, (int)fills.size()});
            i = j;
        } else {
            items.push_back({op0.kind, op0.lane, i, 0, 0, 0, 0, 0});
        }
    }
    char* dev = nullptr;
    if (cudaMalloc(&dev, std::max<size_t>(host.size(), 16)) != cudaSuccess) return SIMOX_E_NOMEM;
    if (cudaMemcpy(dev, host.data(), host.size(), cudaMemcpyHostToDevice) != cudaSuccess) {
        cudaFree(dev);
        return SIMOX_E_CUDA;
    }
    for (const Item& it : items)
        if (it.kind == sx::RecOp::KERNEL && it.smem > 48 * 1024)
            cudaFuncSetAttribute(rec[0].ops[it.pos].fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)it.smem);

    // issue every operation once for all members, on the master (lane 0) and
    // the batch's side stream (lane 1)
    cudaStream_t lane[2] = {b->master, b->side};
    long long launched = 0;
    if (cudaStreamBeginCapture(b->master, cudaStreamCaptureModeThreadLocal) != cudaSuccess) {
        cudaFree(dev);
        return SIMOX_E_CUDA;
    }
    int st = SIMOX_OK;
    for (const Item& it : items) {
        const sx::RecOp& op0 = rec[0].ops[it.pos];
        cudaStream_t s = lane[it.lane];
        switch (it.kind) {
            case sx::RecOp::KERNEL: {
                if (it.blocks == 0) break;
                void* packs = dev + it.off_a;
                void* bstart = dev + it.off_b;
                int n = nsys;
                void* args[3] = {&packs, &bstart, &n};
                if (cudaLaunchKernel(op0.fn, dim3(it.blocks), dim3(op0.threads), args, it.smem, s) != cudaSuccess)
                    st = SIMOX_E_CUDA;
                launched++;
                break;
            }
            case sx::RecOp::MEMSET:
                if (it.count == 0) break;
                batched_fill_kernel<<<it.count, 256, 0, s>>>(reinterpret_cast<const sx::FillItem*>(dev + it.off_a));
                launched++;
                break;
            case sx::RecOp::EV_RECORD: cudaEventRecord(b->lane_ev[op0.tag], s); break;
            case sx::RecOp::EV_WAIT: cudaStreamWaitEvent(s, b->lane_ev[op0.tag], 0); break;
            case sx::RecOp::FFT: {
                // one batched plan per group; a member outside every group runs its own plan
                std::vector<const FftGroup*> done;
                for (int k = 0; k < nsys && !st; k++) {
                    const sx::RecOp& r = rec[k].ops[it.pos];
                    int slot = 0;
                    const FftGroup* g = fft_group_of(pool, r, k, &slot);
                    cufftHandle plan = r.plan;
                    void* in = r.in;
                    void* outp = r.out;
                    if (g) {
                        if (std::find(done.begin(), done.end(), g) != done.end()) continue;
                        done.push_back(g);
                        const bool fwd = r.fft == 0 || r.fft == 2;
                        plan = fwd ? g->r2c : g->c2r;
                        in = fwd ? g->real : g->cplx;
                        outp = fwd ? g->cplx : g->real;
                    }
                    cufftResult fr = cufftSetStream(plan, s);
                    if (fr == CUFFT_SUCCESS) {
                        switch (r.fft) {
                            case 0: fr = cufftExecR2C(plan, (cufftReal*)in, (cufftComplex*)outp); break;
                            case 1: fr = cufftExecC2R(plan, (cufftComplex*)in, (cufftReal*)outp); break;
                            case 2: fr = cufftExecD2Z(plan, (cufftDoubleReal*)in, (cufftDoubleComplex*)outp); break;
                            default: fr = cufftExecZ2D(plan, (cufftDoubleComplex*)in, (cufftDoubleReal*)outp); break;
                        }
                    }
                    if (fr != CUFFT_SUCCESS) st = SIMOX_E_CUDA;
                    launched++;
                }
                break;
            }
            default: break;
        }
        if (st) break;
    }
    cudaGraph_t graph = nullptr;
    const cudaError_t ce = cudaStreamEndCapture(b->master, &graph);
    cudaGetLastError();
    for (auto* c : b->ctx) sx::pme_bind_stream(c);
    cudaGraphExec_t exec = nullptr;
    if (!st && ce == cudaSuccess && graph && cudaGraphInstantiate(&exec, graph, 0) != cudaSuccess) exec = nullptr;
    if (graph) cudaGraphDestroy(graph);
    if (st || !exec) {
        cudaFree(dev);
        return st ? st : SIMOX_E_CUDA;
    }
    out.exec = exec;
    out.tables = dev;
    out.kernels = launched;
    out.mode = SIMOX_BATCH_PER_PASS;
    return SIMOX_OK;
}

// the per-system graph: every member's own launches on its own stream
int capture_per_system(simox_batch* b, const simox_md_opts* o, bool sort, bool estep, simox_batch::G& out) {
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
    out.exec = exec;
    out.kernels = l1 - l0;
    out.mode = SIMOX_BATCH_PER_SYSTEM;
    return SIMOX_OK;
}

bool pool_current(const simox_batch* b) {
    if (b->pool_gens.size() != b->ctx.size()) return false;
    for (size_t k = 0; k < b->ctx.size(); k++)
        if (b->pool_gens[k] != b->ctx[k]->graph_gen) return false;
    return true;
}

int graph_step(simox_batch* b, const simox_md_opts* o, bool sort, bool estep) {
    const unsigned key = 1u | (sort ? 2u : 0u) | (estep ? 4u : 0u);
    simox_batch::G* hit = nullptr;
    for (auto& g : b->graphs)
        if (g.exec && g.key == key && graph_current(b, g, o)) hit = &g;
    if (!hit) {
        simox_batch::G fresh;
        if (b->want_mode == SIMOX_BATCH_PER_PASS && !b->per_pass_failed) {
            if (!pool_current(b)) {
                drop(b);   // the other slot's graph may run on the old buffers
                b->pool.release();
                b->pool_gens.clear();
            }
            if (int st = capture_per_pass(b, o, sort, estep, b->pool, fresh)) return st;
            if (b->pool_gens.empty())
                for (auto* c : b->ctx) b->pool_gens.push_back(c->graph_gen);
            if (!fresh.exec) b->per_pass_failed = true;
        }
        if (!fresh.exec)
            if (int st = capture_per_system(b, o, sort, estep, fresh)) return st;
        simox_batch::G& g = b->graphs[estep ? 1 : 0];
        if (g.exec || g.tables) {
            cudaStreamSynchronize(b->master);
            if (g.exec) cudaGraphExecDestroy(g.exec);
            if (g.tables) cudaFree(g.tables);
        }
        g = fresh;
        g.key = key;
        g.opts.assign(o, o + b->ctx.size());
        g.gens.clear();
        for (auto* c : b->ctx) g.gens.push_back(c->graph_gen);
        hit = &g;
    }
    b->launches += hit->kernels;
    b->last_mode = hit->mode;
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
              cudaStreamCreateWithFlags(&b->side, cudaStreamNonBlocking) == cudaSuccess &&
              cudaEventCreateWithFlags(&b->fork, cudaEventDisableTiming) == cudaSuccess &&
              cudaEventCreateWithFlags(&b->lane_ev[0], cudaEventDisableTiming) == cudaSuccess &&
              cudaEventCreateWithFlags(&b->lane_ev[1], cudaEventDisableTiming) == cudaSuccess &&
              cudaEventCreate(&b->t0) == cudaSuccess && cudaEventCreate(&b->t1) == cudaSuccess;
    b->join.assign(nsys, nullptr);
    for (int k = 0; ok && k < nsys; k++)
        ok = cudaEventCreateWithFlags(&b->join[k], cudaEventDisableTiming) == cudaSuccess;
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
    if (b->side) cudaStreamSynchronize(b->side);
    drop(b);
    b->pool.release();
    for (auto e : b->join)
        if (e) cudaEventDestroy(e);
    for (auto e : b->lane_ev)
        if (e) cudaEventDestroy(e);
    if (b->fork) cudaEventDestroy(b->fork);
    if (b->t0) cudaEventDestroy(b->t0);
    if (b->t1) cudaEventDestroy(b->t1);
    if (b->side) cudaStreamDestroy(b->side);
    if (b->master) cudaStreamDestroy(b->master);
    delete b;
    return SIMOX_OK;
}

extern "C" int simox_batch_set_mode(simox_batch* b, int mode) {
    if (!b || (mode != SIMOX_BATCH_PER_PASS && mode != SIMOX_BATCH_PER_SYSTEM)) return SIMOX_E_ARG;
    cudaSetDevice(b->device);
    if (mode != b->want_mode) drop(b);
    b->want_mode = mode;
    b->per_pass_failed = false;
    return SIMOX_OK;
}

extern "C" int simox_batch_get_mode(simox_batch* b, int* mode) {
    if (!b || !mode) return SIMOX_E_ARG;
    *mode = b->last_mode;
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
