// common.hpp -- shared host-side plumbing of libtblis_b200: error state,
// CUDA checks, the library stream, the stream-ordered device workspace and
// the kernel launch counter.
#pragma once

#include <cuda_runtime.h>

#include <atomic>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <stdexcept>
#include <string>
#include <vector>

#include "../../include/tblis_b200.h"

// opaque configuration object of the C ABI (src/util/basic_types.h:51)
struct tblis_config_s
{
    const char* name;
    int method;        // 1 = FP64 DMMA, 2 = Ozaki INT8, 3 = Ozaki BF16, 4 = TF32 pass, 5 = BF16 pass
    double tolerance;  // normwise relative target
};

namespace tb
{

typedef int64_t i64;

// Error codes recorded as the thread's last error.
enum
{
    TB_OK = 0,
    TB_ERR_ARG = 1,        // malformed labels / shapes
    TB_ERR_TYPE = 2,       // unsupported element type
    TB_ERR_CUDA = 3,       // a CUDA runtime call failed
    TB_ERR_NODEV = 4,      // no CUDA device visible
    TB_ERR_SIZE = 5,       // size beyond a documented limit
    TB_ERR_TIMEOUT = 6,    // a bounded device-side wait gave up
    TB_ERR_BUDGET = 7,     // request exceeds the memory budget
};

struct error : std::runtime_error
{
    int code;
    error(int c, const std::string& msg) : std::runtime_error(msg), code(c) {}
};

void set_last_error(int code, const char* msg);

#define TB_CUDA(call)                                                               \
    do {                                                                            \
        cudaError_t e_ = (call);                                                    \
        if (e_ != cudaSuccess)                                                      \
            throw ::tb::error(::tb::TB_ERR_CUDA, std::string(#call) + ": " +         \
                              cudaGetErrorString(e_));                              \
    } while (0)

#define TB_CHECK(cond, code, msg)                                                   \
    do { if (!(cond)) throw ::tb::error((code), (msg)); } while (0)

// Runs f, converting exceptions into the thread's last error (and aborting
// when TBLIS_B200_ABORT_ON_ERROR=1). Returns the error code.
template <typename F>
int guarded(F&& f)
{
    try
    {
        f();
        return TB_OK;
    }
    catch (const error& e)
    {
        set_last_error(e.code, e.what());
        return e.code;
    }
    catch (const std::exception& e)
    {
        set_last_error(TB_ERR_ARG, e.what());
        return TB_ERR_ARG;
    }
}

// runs one of this library's C entry points from inside another call and
// turns its recorded error into an exception
template <typename F>
void checked(F&& f)
{
    tblis_b200_clear_error();
    f();
    const int c = tblis_b200_last_error();
    if (c) throw error(c, tblis_b200_last_error_string());
}

cudaStream_t current_stream();
void ensure_device();

// kernel launch accounting (every launch of this library's kernels)
extern std::atomic<int64_t> g_kernel_count;
inline void count_launch(int n = 1) { g_kernel_count.fetch_add(n, std::memory_order_relaxed); }

// optional per-kernel device timing: while enabled, a TimedLaunch scope
// around a launch records a CUDA event pair on the launching stream; the
// pairs are read back (and the stream waited for) only on request
extern std::atomic<bool> g_ktimer_on;
void ktimer_push(const char* name, cudaEvent_t a, cudaEvent_t b);
struct TimedLaunch
{
    const char* name;
    cudaStream_t st;
    cudaEvent_t a = nullptr;
    TimedLaunch(const char* n, cudaStream_t s) : name(n), st(s)
    {
        if (g_ktimer_on.load(std::memory_order_relaxed) && cudaEventCreate(&a) == cudaSuccess)
            cudaEventRecord(a, st);
    }
    ~TimedLaunch()
    {
        if (!a) return;
        cudaEvent_t b = nullptr;
        if (cudaEventCreate(&b) == cudaSuccess && cudaEventRecord(b, st) == cudaSuccess) ktimer_push(name, a, b);
        else { cudaEventDestroy(a); if (b) cudaEventDestroy(b); }
    }
};

// checks the launch status right after a kernel launch
inline void check_launch(const char* what)
{
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess)
        throw error(TB_ERR_CUDA, std::string("launch of ") + what + ": " + cudaGetErrorString(e));
    count_launch();
}

// Stream-ordered device allocation from the device's default memory pool
// (the GPU counterpart of TBLIS's MemoryPool, src/memory/memory_pool.hpp:18-166).
struct dbuf
{
    void* ptr = nullptr;
    size_t bytes = 0;
    cudaStream_t stream = 0;

    dbuf() {}
    dbuf(size_t n, cudaStream_t s) : bytes(n), stream(s)
    {
        if (n) TB_CUDA(cudaMallocAsync(&ptr, n, s));
    }
    dbuf(const dbuf&) = delete;
    dbuf& operator=(const dbuf&) = delete;
    dbuf(dbuf&& o) noexcept : ptr(o.ptr), bytes(o.bytes), stream(o.stream) { o.ptr = nullptr; o.bytes = 0; }
    dbuf& operator=(dbuf&& o) noexcept
    {
        release();
        ptr = o.ptr; bytes = o.bytes; stream = o.stream;
        o.ptr = nullptr; o.bytes = 0;
        return *this;
    }
    ~dbuf() { release(); }
    void release()
    {
        if (ptr) cudaFreeAsync(ptr, stream);
        ptr = nullptr; bytes = 0;
    }
    template <typename T> T* as() const { return static_cast<T*>(ptr); }
};

// where a pointer lives
enum mem_kind { MEM_DEVICE, MEM_HOST };
mem_kind pointer_kind(const void* p);

} // namespace tb
