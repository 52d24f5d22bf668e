// common.cuh -- shared device/host helpers of the B200 TeaLeaf kernel suites.
//
// * Error handling with the reference's contract: a fatal error prints and
//   calls exit(1) like die() (2d/shared.c:97-111), unless the caller switched
//   the library to "record" mode, where the first error is kept and every
//   later call returns early until the host reads it.
// * Deterministic reductions: every block reduces its per-thread values with
//   warp shuffles in a fixed tree, writes one partial per value, and the last
//   block to finish (atomic ticket) reduces the partials in a fixed order and
//   publishes the result to device memory and to a mapped pinned host slot.
//   The result depends only on the launch shape, never on block scheduling,
//   so iteration counts are reproducible run to run.
#pragma once

#include <cuda_runtime.h>
#include <cstdarg>
#include <vector>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>

// Hidden: each shared library keeps its own error state and helpers.
namespace tl __attribute__((visibility("hidden"))) {

constexpr int kWarp = 32;

// ---------------------------------------------------------------- errors --
struct ErrorState {
    int mode = 0;          // 0: exit(1) on error, 1: record and return
    int code = 0;          // first recorded error (0: none)
    char msg[512] = {0};
};

inline ErrorState& error_state()
{
    static ErrorState st;  // one per shared library (hidden visibility)
    return st;
}

inline void fail(int code, const char* fmt, ...)
{
    ErrorState& st = error_state();
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof(buf), fmt, ap);
    va_end(ap);
    if (st.mode == 0) {
        fprintf(stdout, "\x1b[31m\nError in the B200 kernel suite:\x1b[0m \n%s\n", buf);
        fflush(stdout);
        exit(1);
    }
    if (st.code == 0) {
        st.code = code;
        snprintf(st.msg, sizeof(st.msg), "%s", buf);
    }
}

inline bool failed() { return error_state().code != 0; }

inline int take_error(char* msg, int len)
{
    ErrorState& st = error_state();
    int c = st.code;
    if (msg && len > 0) snprintf(msg, (size_t)len, "%s", st.msg);
    st.code = 0;
    st.msg[0] = 0;
    return c;
}

inline bool cuda_ok(cudaError_t e, const char* what, const char* file, int line)
{
    if (e == cudaSuccess) return true;
    fail((int)e, "CUDA error %d (%s) in %s at %s:%d", (int)e, cudaGetErrorString(e), what, file, line);
    return false;
}

#define TL_CUDA(call) ::tl::cuda_ok((call), #call, __FILE__, __LINE__)
#define TL_LAUNCHED(name) ::tl::cuda_ok(cudaGetLastError(), name, __FILE__, __LINE__)

inline int ceil_div(long a, long b) { return (int)((a + b - 1) / b); }

// -------------------------------------------------------------- profiler --
// Device-time profile of every kernel launch, by kernel name: a CUDA event
// pair brackets each launch on the launching stream, and pairs are resolved
// into milliseconds at the next host synchronisation (or on read), so
// profiling adds no synchronisation of its own. The B200 counterpart of the
// reference's per-call START_PROFILING/STOP_PROFILING (2d/profiler.h:49-71).
class Profiler {
public:
    static constexpr int kMaxKernels = 64;
    bool on = false;
    long long launches = 0;   // every launch, counted whether or not timing is on
    const char* names[kMaxKernels] = {nullptr};
    long calls[kMaxKernels] = {0};
    double ms[kMaxKernels] = {0.0};

    int id_of(const char* name)
    {
        for (int i = 0; i < kMaxKernels; ++i) {
            if (names[i] == name || (names[i] && strcmp(names[i], name) == 0)) return i;
            if (!names[i]) {
                names[i] = name;
                return i;
            }
        }
        return kMaxKernels - 1;
    }
    void begin(cudaStream_t st, const char* name)
    {
        ++launches;
        if (!on) return;
        Pending p;
        p.id = id_of(name);
        p.a = take();
        p.b = take();
        cudaEventRecord(p.a, st);
        pending_.push_back(p);
    }
    void end(cudaStream_t st)
    {
        if (!on || pending_.empty()) return;
        cudaEventRecord(pending_.back().b, st);
    }
    // Call after the stream was synchronised (or to force: synchronises events).
    void resolve()
    {
        for (Pending& p : pending_) {
            cudaEventSynchronize(p.b);
            float t = 0.f;
            if (cudaEventElapsedTime(&t, p.a, p.b) == cudaSuccess) {
                ms[p.id] += t;
                calls[p.id] += 1;
            }
            pool_.push_back(p.a);
            pool_.push_back(p.b);
        }
        pending_.clear();
    }
    void reset()
    {
        resolve();
        for (int i = 0; i < kMaxKernels; ++i) {
            calls[i] = 0;
            ms[i] = 0.0;
        }
    }
    ~Profiler()
    {
        for (cudaEvent_t e : pool_) cudaEventDestroy(e);
    }

private:
    struct Pending {
        int id;
        cudaEvent_t a, b;
    };
    std::vector<Pending> pending_;
    std::vector<cudaEvent_t> pool_;
    cudaEvent_t take()
    {
        if (!pool_.empty()) {
            cudaEvent_t e = pool_.back();
            pool_.pop_back();
            return e;
        }
        cudaEvent_t e;
        cudaEventCreate(&e);
        return e;
    }
};

// ------------------------------------------------------------ reductions --
// Scratch of one reduction slot set. partials: capacity >= blocks * kMaxSums.
constexpr int kMaxSums = 4;

struct ReduceSlots {
    double* partials;        // device, [blocks * nsum]
    unsigned int* ticket;    // device, one counter, 0 between launches
    double* out_dev;         // device, [kMaxSums]
    double* out_host;        // mapped pinned host memory, [kMaxSums] (device-visible pointer)
};

__device__ __forceinline__ double warp_sum(double v)
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    return v;  // lane 0
}

// Linear thread index of 1-, 2- or 3-D blocks (blockDim.x a multiple of 32
// or the only dimension, so warps are contiguous runs of it).
__device__ __forceinline__ int linear_tid()
{
    return threadIdx.x + blockDim.x * (threadIdx.y + blockDim.y * threadIdx.z);
}

// Block sum of N values; thread 0 holds the sums in v afterwards.
template <int N, int BLOCK>
__device__ __forceinline__ void block_sum(double (&v)[N], double (*smem)[BLOCK / kWarp])
{
    const int tid = linear_tid();
    const int lane = tid & (kWarp - 1);
    const int warp = tid / kWarp;
#pragma unroll
    for (int r = 0; r < N; ++r) v[r] = warp_sum(v[r]);
    if (lane == 0) {
#pragma unroll
        for (int r = 0; r < N; ++r) smem[r][warp] = v[r];
    }
    __syncthreads();
    if (warp == 0) {
#pragma unroll
        for (int r = 0; r < N; ++r) {
            double t = (lane < BLOCK / kWarp) ? smem[r][lane] : 0.0;
            v[r] = warp_sum(t);
        }
    }
}

// Grid-wide deterministic sum of N per-thread values (1-D block index `bid`
// of `nblocks`). The last block publishes the totals; `finish` (optional)
// runs in thread 0 of that block with the totals, for fused scalar updates.
struct NoFinish {
    __device__ void operator()(const double*) const {}
};

template <int N, int BLOCK, typename Finish = NoFinish>
__device__ __forceinline__ void grid_sum(double (&v)[N], const ReduceSlots& s, int bid, int nblocks,
                                         const Finish& finish = Finish())
{
    __shared__ double smem[N][BLOCK / kWarp];
    __shared__ bool last;
    const int tid = linear_tid();
    block_sum<N, BLOCK>(v, smem);
    if (tid == 0) {
#pragma unroll
        for (int r = 0; r < N; ++r) s.partials[(long)bid * N + r] = v[r];
        __threadfence();
        unsigned int prev = atomicAdd(s.ticket, 1u);
        last = (prev == (unsigned int)(nblocks - 1));
    }
    __syncthreads();
    if (!last) return;
    __threadfence();
    double t[N];
#pragma unroll
    for (int r = 0; r < N; ++r) t[r] = 0.0;
    for (int b = tid; b < nblocks; b += BLOCK) {
#pragma unroll
        for (int r = 0; r < N; ++r) t[r] += __ldcg(&s.partials[(long)b * N + r]);
    }
    __syncthreads();  // smem reuse
    block_sum<N, BLOCK>(t, smem);
    if (tid == 0) {
#pragma unroll
        for (int r = 0; r < N; ++r) {
            s.out_dev[r] = t[r];
            if (s.out_host) s.out_host[r] = t[r];
        }
        finish(t);
        *s.ticket = 0u;
    }
}

}  // namespace tl
