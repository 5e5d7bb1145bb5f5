// Host-only check of pb::DevArena (prism_b200/csrc/common.h), the allocator of
// the AMG hierarchy: the CUDA entry points it calls are replaced by fakes that
// hand out host memory, so the bump / mark / rewind / reset logic runs without
// a GPU. Checked for random build sequences shaped like a hierarchy build
// (persistent buffers, intermediates rewound per level, rebuilds):
//   * every buffer is 256-byte aligned and lies inside one chunk;
//   * no two live buffers overlap;
//   * chunks grow geometrically (few pool calls per build);
//   * the destructor returns every chunk, on the device the arena took them on,
//     and leaves the caller's current device current.
#include "../../prism_b200/csrc/common.h"

#include <cstdio>
#include <map>
#include <random>

namespace {
std::map<char*, size_t> g_chunks;
std::map<char*, int> g_chunk_device;
long g_pool_calls = 0;
int g_failures = 0;
int g_device = 0;  // the fake current device

void check(bool ok, const char* what) {
    if (!ok && g_failures++ < 10) std::fprintf(stderr, "FAILED: %s\n", what);
}
}  // namespace

extern "C" {
cudaError_t cudaMallocFromPoolAsync(void** p, size_t size, cudaMemPool_t, cudaStream_t) {
    *p = std::aligned_alloc(256, (size + 255) / 256 * 256);
    g_chunks[static_cast<char*>(*p)] = size;
    g_chunk_device[static_cast<char*>(*p)] = g_device;
    ++g_pool_calls;
    return cudaSuccess;
}
cudaError_t cudaFree(void* p) {
    check(g_chunks.erase(static_cast<char*>(p)) == 1, "free of an unknown chunk");
    check(g_chunk_device[static_cast<char*>(p)] == g_device, "chunk freed with its own device current");
    g_chunk_device.erase(static_cast<char*>(p));
    std::free(p);
    return cudaSuccess;
}
cudaError_t cudaDeviceSynchronize() { return cudaSuccess; }
cudaError_t cudaGetDevice(int* d) {
    *d = g_device;
    return cudaSuccess;
}
cudaError_t cudaSetDevice(int d) {
    g_device = d;
    return cudaSuccess;
}
cudaError_t cudaMemPoolCreate(cudaMemPool_t* p, const cudaMemPoolProps*) {
    *p = reinterpret_cast<cudaMemPool_t>(uintptr_t(1));
    return cudaSuccess;
}
cudaError_t cudaMemPoolSetAttribute(cudaMemPool_t, cudaMemPoolAttr, void*) { return cudaSuccess; }
cudaError_t cudaGetLastError() { return cudaSuccess; }
const char* cudaGetErrorString(cudaError_t) { return "fake"; }
cudaError_t cudaMemsetAsync(void*, int, size_t, cudaStream_t) { return cudaSuccess; }
cudaError_t cudaMemcpyAsync(void*, const void*, size_t, cudaMemcpyKind, cudaStream_t) { return cudaSuccess; }
}

int main() {
    std::mt19937_64 rng(7);
    long builds = 0;
    for (int trial = 0; trial < 200; ++trial) {
        // every third arena lives on device 1 and is destroyed while device 0 is current
        g_device = (trial % 3 == 0) ? 1 : 0;
        {
            pb::DevArena arena;
            struct Live {
                const char* p;
                size_t bytes;
            };
            std::vector<Live> live;
            auto take = [&](size_t count) {
                const double* p = arena.take<double>(count, nullptr);
                if (!count) {
                    check(p == nullptr, "empty request returns null");
                    return;
                }
                const char* c = reinterpret_cast<const char*>(p);
                check((reinterpret_cast<uintptr_t>(c) & 255) == 0, "256-byte alignment");
                bool inside = false;
                for (auto& [base, size] : g_chunks)
                    if (c >= base && c + count * sizeof(double) <= base + size) inside = true;
                check(inside, "buffer inside a chunk");
                for (auto& l : live)
                    check(c + count * sizeof(double) <= l.p || l.p + l.bytes <= c, "live buffers do not overlap");
                live.push_back({c, count * sizeof(double)});
            };
            for (int rebuild = 0; rebuild < 3; ++rebuild, ++builds) {
                live.clear();
                arena.reset();
                size_t n = 1 + rng() % 4000000;
                const int levels = 1 + int(rng() % 8);
                take(n);
                for (int l = 0; l < levels; ++l) {
                    take(n / 2);  // persistent (aggregate map)
                    const pb::DevArena::Mark m = arena.mark();
                    const size_t keep = live.size();
                    for (int k = 0; k < 9; ++k) take(rng() % (n + 1));  // intermediates
                    live.resize(keep);
                    arena.rewind(m);
                    for (int k = 0; k < 9; ++k) take(rng() % (n + 1));  // next level
                    n = n / 4 + 1;
                }
            }
            g_device = 0;
        }
        check(g_chunks.empty(), "destructor returns every chunk");
        check(g_device == 0, "destructor restores the current device");
    }
    const double per_build = double(g_pool_calls) / double(builds);
    check(per_build < 4.0, "few pool calls per build");
    std::printf("arena: %ld builds, %.2f pool calls per build, %d failures\n", builds, per_build, g_failures);
    return g_failures ? 1 : 0;
}
