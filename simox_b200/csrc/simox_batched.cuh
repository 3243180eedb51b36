// simox_batched.cuh -- one launch of a kernel over the blocks of many
// independent systems (no counterpart in the reference, which runs one
// system per process).
//
// A kernel on the MD step path is written as a body, a device function that
// takes its block coordinates as a Blk argument instead of reading blockIdx
// and gridDim.  The named __global__ kernel runs the body over its own launch;
// batched_kernel runs it over a work list: block b of a batched launch
// belongs to the system s with bstart[s] <= b < bstart[s+1], takes that
// system's arguments from a device table of argument packs and runs as block
// b - bstart[s] of a grid of bstart[s+1] - bstart[s] blocks.  A body is the
// same code in both, so a system advanced in a batch computes exactly what it
// computes alone.
//
// While a batch records a context's step (simox_ctx::rec set), launch_k,
// memset_async, event_record, stream_wait and the FFT calls write the step
// down as a list of operations instead of issuing them; the batch checks that
// every system's list has the same sequence and issues each operation once
// for all systems.
#pragma once

#include <cstring>
#include <type_traits>
#include <utility>
#include <vector>

namespace sx {

struct Blk {
    int x;   // block index within the system's grid
    int n;   // the system's block count
};
__device__ __forceinline__ Blk own_blk() { return Blk{(int)blockIdx.x, (int)gridDim.x}; }

// A kernel's arguments as one aggregate, laid out the same by the host and
// the device compiler; call<F>(blk) runs F(blk, arguments...).
template <typename... K>
struct Pack;
template <>
struct Pack<> {
    template <auto F, typename... D>
    __device__ __forceinline__ void call(Blk b, const D&... d) const {
        F(b, d...);
    }
};
template <typename H, typename... R>
struct Pack<H, R...> {
    H h;
    Pack<R...> r;
    template <auto F, typename... D>
    __device__ __forceinline__ void call(Blk b, const D&... d) const {
        r.template call<F>(b, d..., h);
    }
};
inline Pack<> make_pack() { return {}; }
template <typename H, typename... R>
inline Pack<H, R...> make_pack(H h, R... r) {
    return Pack<H, R...>{h, make_pack(r...)};
}

template <int T, int M, auto Body, typename... K>
__global__ void __launch_bounds__(T, M)
    batched_kernel(const Pack<K...>* __restrict__ packs, const int* __restrict__ bstart, int nsys) {
    const int b = (int)blockIdx.x;
    int lo = 0, hi = nsys;   // bstart[lo] <= b < bstart[hi]
    while (hi - lo > 1) {
        const int mid = (lo + hi) >> 1;
        if (__ldg(bstart + mid) <= b) lo = mid;
        else hi = mid;
    }
    const int b0 = __ldg(bstart + lo);
    // the arguments stay in the table: a body reads the fields it uses
    packs[lo].template call<Body>(Blk{b - b0, __ldg(bstart + lo + 1) - b0});
}

// byte fills of a batched step, one block per range
struct FillItem {
    void* p;
    unsigned long long bytes;
    int value;
    int pad_;
};

// One operation of a recorded step.
struct RecOp {
    enum Kind : int { KERNEL = 0, MEMSET, EV_RECORD, EV_WAIT, FFT };
    int kind = KERNEL;
    int lane = 0;                    // 0: the context's stream, 1: its side stream
    // KERNEL: the batched instance of the body, its block size, the system's
    // grid and dynamic shared memory, the argument pack's bytes
    const void* fn = nullptr;
    int threads = 0;
    unsigned grid = 0;
    size_t smem = 0;
    std::vector<unsigned char> args;
    // MEMSET
    void* ptr = nullptr;
    int value = 0;
    size_t bytes = 0;
    // EV_RECORD / EV_WAIT: 0 the fork event, 1 the join event
    int tag = 0;
    // FFT: 0 R2C, 1 C2R, 2 D2Z, 3 Z2D of plan from in to out
    cufftHandle plan = 0;
    int fft = 0;
    void* in = nullptr;
    void* out = nullptr;
    const char* name = nullptr;
};

struct Recorder {
    cudaStream_t main = nullptr, side = nullptr;
    std::vector<RecOp> ops;
    bool bad = false;   // an operation a batch cannot issue for all systems
    int lane(cudaStream_t s) {
        if (s == main) return 0;
        if (s == side) return 1;
        bad = true;
        return 0;
    }
};

// Launch `single` (or record the launch): Body is its body, T its block size
// and M its minimum resident blocks per SM (the batched instance's bounds).
template <int T, int M, auto Body, typename... K, typename... A>
inline void launch_k(simox_ctx* c, void (*single)(K...), unsigned grid, size_t smem, cudaStream_t s, A... a) {
    if (c->rec) {
        static_assert(std::is_trivially_copyable<Pack<K...>>::value, "kernel arguments must be plain data");
        static_assert(alignof(Pack<K...>) <= 256, "argument tables are 256-byte aligned");
        const Pack<K...> pk = make_pack(K(a)...);
        RecOp op;
        op.kind = RecOp::KERNEL;
        op.lane = c->rec->lane(s);
        op.fn = (const void*)&batched_kernel<T, M, Body, K...>;
        op.threads = T;
        op.grid = grid;
        op.smem = smem;
        op.args.resize(sizeof(pk));
        std::memcpy(op.args.data(), &pk, sizeof(pk));
        c->rec->ops.push_back(std::move(op));
        return;
    }
    single<<<grid, T, smem, s>>>(K(a)...);
}

inline void memset_async(simox_ctx* c, void* p, int value, size_t bytes, cudaStream_t s) {
    if (c->rec) {
        RecOp op;
        op.kind = RecOp::MEMSET;
        op.lane = c->rec->lane(s);
        op.ptr = p;
        op.value = value;
        op.bytes = bytes;
        c->rec->ops.push_back(std::move(op));
        return;
    }
    cudaMemsetAsync(p, value, bytes, s);
}

inline int event_tag(simox_ctx* c, cudaEvent_t e) {
    if (e == c->ev_fork) return 0;
    if (e == c->ev_join) return 1;
    c->rec->bad = true;
    return 0;
}

inline void event_record(simox_ctx* c, cudaEvent_t e, cudaStream_t s) {
    if (c->rec) {
        RecOp op;
        op.kind = RecOp::EV_RECORD;
        op.lane = c->rec->lane(s);
        op.tag = event_tag(c, e);
        c->rec->ops.push_back(std::move(op));
        return;
    }
    cudaEventRecord(e, s);
}

inline void stream_wait(simox_ctx* c, cudaStream_t s, cudaEvent_t e) {
    if (c->rec) {
        RecOp op;
        op.kind = RecOp::EV_WAIT;
        op.lane = c->rec->lane(s);
        op.tag = event_tag(c, e);
        c->rec->ops.push_back(std::move(op));
        return;
    }
    cudaStreamWaitEvent(s, e, 0);
}

}  // namespace sx
