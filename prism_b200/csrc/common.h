// common.h -- error handling, device buffers and launch helpers shared by the
// host runtime and the sm_100a kernels of libprism_b200.
#pragma once

#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <stdexcept>
#include <string>
#include <utility>
#include <vector>

#include "../../include/prism_b200.h"

namespace pb {

// Status-carrying exception used inside the library; converted to an int
// status at the C-ABI boundary (nothing is thrown across it).
struct Error {
    int status;
    std::string msg;
};
[[noreturn]] inline void fail(int status, const std::string& msg) { throw Error{status, msg}; }

inline void cudaCheck(cudaError_t e, const char* what) {
    if (e != cudaSuccess) {
        cudaGetLastError();
        if (e == cudaErrorMemoryAllocation) fail(PRISM_OUT_OF_MEMORY, std::string(what) + ": " + cudaGetErrorString(e));
        fail(PRISM_CUDA_ERROR, std::string(what) + ": " + cudaGetErrorString(e));
    }
}
#define PB_CUDA(call) ::pb::cudaCheck((call), #call)
#define PB_LAUNCH(what) ::pb::cudaCheck(cudaGetLastError(), what)

// Owning device allocation (cudaMalloc / cudaFree).
template <typename T>
struct DevBuf {
    T* p = nullptr;
    size_t n = 0;
    DevBuf() = default;
    explicit DevBuf(size_t count) { alloc(count); }
    DevBuf(const DevBuf&) = delete;
    DevBuf& operator=(const DevBuf&) = delete;
    DevBuf(DevBuf&& o) noexcept : p(o.p), n(o.n) { o.p = nullptr; o.n = 0; }
    DevBuf& operator=(DevBuf&& o) noexcept {
        if (this != &o) { release(); p = o.p; n = o.n; o.p = nullptr; o.n = 0; }
        return *this;
    }
    ~DevBuf() { release(); }
    void alloc(size_t count) {
        release();
        n = count;
        if (count) PB_CUDA(cudaMalloc(&p, count * sizeof(T)));
    }
    void release() {
        if (p) cudaFree(p);
        p = nullptr;
        n = 0;
    }
    void upload(const T* h, size_t count, cudaStream_t s) {
        if (count > n) fail(PRISM_INTERNAL, "upload beyond allocation");
        if (count) PB_CUDA(cudaMemcpyAsync(p, h, count * sizeof(T), cudaMemcpyHostToDevice, s));
    }
    void upload(const std::vector<T>& h, cudaStream_t s) {
        if (h.size() != n) alloc(h.size());
        upload(h.data(), h.size(), s);
    }
    void download(T* h, size_t count, cudaStream_t s) const {
        if (count > n) fail(PRISM_INTERNAL, "download beyond allocation");
        if (count) PB_CUDA(cudaMemcpyAsync(h, p, count * sizeof(T), cudaMemcpyDeviceToHost, s));
    }
    void zero(cudaStream_t s) {
        if (n) PB_CUDA(cudaMemsetAsync(p, 0, n * sizeof(T), s));
    }
    explicit operator bool() const { return p != nullptr; }
};

// Non-owning slice of a device allocation (several arrays carved from one
// allocation, which costs one cudaMalloc instead of one per array).
template <typename T>
struct DevSlice {
    T* p = nullptr;
    size_t n = 0;
    void zero(cudaStream_t s) {
        if (n) PB_CUDA(cudaMemsetAsync(p, 0, n * sizeof(T), s));
    }
    void download(T* h, size_t count, cudaStream_t s) const {
        if (count > n) fail(PRISM_INTERNAL, "download beyond allocation");
        if (count) PB_CUDA(cudaMemcpyAsync(h, p, count * sizeof(T), cudaMemcpyDeviceToHost, s));
    }
    explicit operator bool() const { return p != nullptr; }
};

// Library-owned stream-ordered memory pool of the current device, for the
// temporaries and hierarchies of setup phases. A cudaMalloc / cudaFree pair
// costs milliseconds here, so blocks freed to the pool stay reserved (up to
// SCRATCH_KEEP bytes) and are handed to later allocations without a call into
// the driver.
constexpr uint64_t SCRATCH_KEEP = uint64_t(2) << 30;
inline cudaMemPool_t scratchPool() {
    static cudaMemPool_t pools[64] = {};
    int dev = 0;
    PB_CUDA(cudaGetDevice(&dev));
    if (dev < 0 || dev >= 64) fail(PRISM_INTERNAL, "device index out of range");
    if (!pools[dev]) {
        cudaMemPoolProps props = {};
        props.allocType = cudaMemAllocationTypePinned;
        props.location.type = cudaMemLocationTypeDevice;
        props.location.id = dev;
        PB_CUDA(cudaMemPoolCreate(&pools[dev], &props));
        uint64_t keep = SCRATCH_KEEP;
        PB_CUDA(cudaMemPoolSetAttribute(pools[dev], cudaMemPoolAttrReleaseThreshold, &keep));
    }
    return pools[dev];
}

// Temporary device buffer in stream order on stream s (scratchPool()).
template <typename T>
struct TmpBuf {
    T* p = nullptr;
    size_t n = 0;
    cudaStream_t s = nullptr;
    TmpBuf(size_t count, cudaStream_t st) : n(count), s(st) {
        if (count)
            PB_CUDA(cudaMallocFromPoolAsync(reinterpret_cast<void**>(&p), count * sizeof(T), scratchPool(), s));
    }
    TmpBuf(const TmpBuf&) = delete;
    TmpBuf& operator=(const TmpBuf&) = delete;
    ~TmpBuf() {
        if (p) cudaFreeAsync(p, s);
    }
};

// Device memory handed out in bump order from a few large chunks of
// scratchPool() and returned all at once, for objects made of many buffers
// (the AMG hierarchy): one pool call per chunk instead of one cudaMalloc per
// buffer. Chunks grow geometrically (at least MIN_CHUNK, at least the total so
// far). mark()/rewind() give back everything taken after the mark, for
// intermediates of a build; reset() gives back everything. Chunks are
// allocated in order on the stream of the call, so work on that stream may use
// them at once; the destructor waits for the device before freeing them.
class DevArena {
public:
    struct Mark {
        size_t chunk = 0, off = 0;
    };
    DevArena() = default;
    DevArena(const DevArena&) = delete;
    DevArena& operator=(const DevArena&) = delete;
    // drains and frees on the device the chunks were taken on, whichever device is
    // current at destruction (several meshes may live on several GPUs of one process)
    ~DevArena() {
        if (chunks_.empty()) return;
        int cur = device_;
        cudaGetDevice(&cur);
        if (cur != device_) cudaSetDevice(device_);
        cudaDeviceSynchronize();
        for (auto& c : chunks_) cudaFree(c.p);
        if (cur != device_) cudaSetDevice(cur);
    }
    template <typename T>
    T* take(size_t count, cudaStream_t s) {
        if (!count) return nullptr;
        const size_t bytes = (count * sizeof(T) + ALIGN - 1) & ~(ALIGN - 1);
        for (; cur_ < chunks_.size(); ++cur_, off_ = 0)
            if (off_ + bytes <= chunks_[cur_].size) {
                char* p = chunks_[cur_].p + off_;
                off_ += bytes;
                return reinterpret_cast<T*>(p);
            }
        size_t size = std::max(std::max(bytes, MIN_CHUNK), total_);
        if (chunks_.empty()) PB_CUDA(cudaGetDevice(&device_));
        char* p = nullptr;
        PB_CUDA(cudaMallocFromPoolAsync(reinterpret_cast<void**>(&p), size, scratchPool(), s));
        chunks_.push_back({p, size});
        total_ += size;
        cur_ = chunks_.size() - 1;
        off_ = bytes;
        return reinterpret_cast<T*>(p);
    }
    Mark mark() const { return {cur_, off_}; }
    // bytes taken (up to the current position) and bytes held in chunks
    size_t used() const {
        size_t u = off_;
        for (size_t i = 0; i < cur_ && i < chunks_.size(); ++i) u += chunks_[i].size;
        return chunks_.empty() ? 0 : u;
    }
    size_t reserved() const { return total_; }
    void rewind(const Mark& m) {
        cur_ = m.chunk;
        off_ = m.off;
    }
    void reset() { rewind(Mark{}); }

private:
    struct Chunk {
        char* p;
        size_t size;
    };
    static constexpr size_t ALIGN = 256;
    static constexpr size_t MIN_CHUNK = size_t(2) << 20;
    std::vector<Chunk> chunks_;
    size_t cur_ = 0, off_ = 0, total_ = 0;
    int device_ = 0;  // device current when the first chunk was taken
};

// A buffer inside a DevArena: the arena owns the memory, so release() only
// forgets it.
template <typename T>
struct ArenaBuf {
    T* p = nullptr;
    size_t n = 0;
    void alloc(DevArena& a, size_t count, cudaStream_t s) {
        p = a.take<T>(count, s);
        n = count;
    }
    void release() {
        p = nullptr;
        n = 0;
    }
    void zero(cudaStream_t s) {
        if (n) PB_CUDA(cudaMemsetAsync(p, 0, n * sizeof(T), s));
    }
    explicit operator bool() const { return p != nullptr; }
};

// Number of kernels this library has launched (read by the profiling window).
inline std::atomic<long long>& launchCounter() {
    static std::atomic<long long> c{0};
    return c;
}
inline void countLaunch() { launchCounter().fetch_add(1, std::memory_order_relaxed); }
// Number of solves and steps this library has run as one CUDA graph launch.
inline std::atomic<long long>& graphLaunchCounter() {
    static std::atomic<long long> c{0};
    return c;
}

inline int ceil_div(int64_t a, int64_t b) { return (int)((a + b - 1) / b); }

// PRISM_VERBOSE=1 in the environment: solver diagnostics on stderr
// (hierarchy sizes, per-solve timings and iteration counts).
inline bool verbose() {
    static const bool v = [] {
        const char* e = std::getenv("PRISM_VERBOSE");
        return e && e[0] && e[0] != '0';
    }();
    return v;
}
// PRISM_VERBOSE=2: also every reliable update and restart of the mixed-precision solver
inline int verboseLevel() {
    static const int v = [] {
        const char* e = std::getenv("PRISM_VERBOSE");
        return e && e[0] ? std::atoi(e) : 0;
    }();
    return v;
}

// Programmatic dependent launch (sm_90 and later). Kernels of the solver
// iteration are launched with launchPdl(): the next kernel in the stream may be
// scheduled while this one drains, and waits in pdlEnter() until this one has
// completed and its writes are visible. PRISM_NO_PDL=1 launches them plainly.
inline bool pdlEnabled() {
    static const bool on = [] {
        const char* e = std::getenv("PRISM_NO_PDL");
        return !(e && e[0] && e[0] != '0');
    }();
    return on;
}
template <typename... KArgs, typename... Args>
void launchPdl(void (*kernel)(KArgs...), int grid, int block, cudaStream_t s, Args... args) {
    cudaLaunchConfig_t cfg{};
    cfg.gridDim = dim3((unsigned)grid);
    cfg.blockDim = dim3((unsigned)block);
    cfg.dynamicSmemBytes = 0;
    cfg.stream = s;
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    at[0].val.programmaticStreamSerializationAllowed = pdlEnabled() ? 1 : 0;
    cfg.attrs = at;
    cfg.numAttrs = 1;
    PB_CUDA(cudaLaunchKernelEx(&cfg, kernel, static_cast<KArgs>(args)...));
    countLaunch();
}
#ifdef __CUDACC__
// First statement of a kernel launched by launchPdl(): release the next kernel's
// launch, then wait for the previous kernel (no-ops without the attribute).
__device__ __forceinline__ void pdlEnter() {
    asm volatile("griddepcontrol.launch_dependents;\n" ::: "memory");
    asm volatile("griddepcontrol.wait;\n" ::: "memory");
}
#endif

constexpr double EPSILON = 2.220446049250313080847263336181640625e-16; // std::numeric_limits<double>::epsilon()
constexpr int SLICE = 32;  // SELL slice height: one warp of rows
constexpr int NUM_SMS = 148;

}  // namespace pb
