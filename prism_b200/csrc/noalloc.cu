// noalloc.cu -- a Jacobi sweep that allocates no memory, for callers that cannot
// call cudaMalloc.
//
// Some callers cannot allocate device memory at the point where they need a
// solver step: solvers embedded in a host application that owns a fixed
// device-memory budget and forbids allocation after start-up, or a time-stepping
// loop where a cudaMalloc/cudaFree pair would synchronize the device every step.
// prism_jacobi_step_noalloc gives them one Jacobi sweep, x <- x + D^-1 (b - A x),
// on a CSR matrix they already hold in device memory.
//
// The sweep has to be computed out of place (every row reads the old x of its
// neighbours), so it needs an n-double scratch vector. Here that scratch is a
// file-scope __device__ array of PRISM_NOALLOC_MAX_ROWS doubles (8 MiB), which
// every GPU that loads the library holds until the process exits. Host code
// cannot use the array's name as a device address (on the host it is only a
// shadow symbol), so its device address is looked up once per device with
// cudaGetSymbolAddress, on the first call made with that device current.
#include <mutex>

#include "common.h"

namespace pb {

namespace {

static __device__ __align__(256) double g_jacobi_scratch[PRISM_NOALLOC_MAX_ROWS];

constexpr int kMaxDevices = 64;
std::mutex g_scratch_mutex;
double* g_scratch_ptr[kMaxDevices] = {};

// Device address of the scratch array for the current device (set-up on first use).
double* scratchAddress() {
    int dev = 0;
    PB_CUDA(cudaGetDevice(&dev));
    if (dev < 0 || dev >= kMaxDevices) fail(PRISM_INTERNAL, "device ordinal out of range");
    std::lock_guard<std::mutex> lock(g_scratch_mutex);
    if (!g_scratch_ptr[dev]) {
        void* p = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&p, g_jacobi_scratch);
        if (e != cudaSuccess || p == nullptr) {
            cudaGetLastError();
            fail(PRISM_CUDA_ERROR, std::string("cudaGetSymbolAddress(jacobi scratch): ") + cudaGetErrorString(e));
        }
        g_scratch_ptr[dev] = static_cast<double*>(p);
    }
    return g_scratch_ptr[dev];
}

// scratch[i] = x[i] + (1 / a_ii) (b[i] - sum_j a_ij x_j)   (numerics/jacobi.cpp:5-9)
// One warp per row. A row without a diagonal entry has a_ii = 0, so 1 / a_ii = inf as in
// the reference's A.diagonal().cwiseInverse().
__global__ void __launch_bounds__(256) jacobi_csr_kernel(int n, const int* __restrict__ rowptr,
                                                         const int* __restrict__ col,
                                                         const double* __restrict__ val,
                                                         const double* __restrict__ b,
                                                         const double* __restrict__ x, double* __restrict__ out) {
    const int row = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (row >= n) return;
    double sum = 0.0, diag = 0.0;
    for (int k = rowptr[row] + lane; k < rowptr[row + 1]; k += 32) {
        const int j = col[k];
        sum += val[k] * x[j];
        if (j == row) diag += val[k];
    }
    for (int o = 16; o > 0; o >>= 1) {
        sum += __shfl_down_sync(0xffffffffu, sum, o);
        diag += __shfl_down_sync(0xffffffffu, diag, o);
    }
    if (lane == 0) out[row] = x[row] + (1.0 / diag) * (b[row] - sum);
}

__global__ void copy_kernel(int n, const double* __restrict__ src, double* __restrict__ dst) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) dst[i] = src[i];
}

}  // namespace

void jacobiStepNoAlloc(int64_t n, const int32_t* rowptr, const int32_t* col, const double* values, const double* b,
                       double* x, cudaStream_t stream) {
    if (n <= 0 || !rowptr || !col || !values || !b || !x) fail(PRISM_BAD_ARG, "prism_jacobi_step_noalloc: bad argument");
    if (n > PRISM_NOALLOC_MAX_ROWS)
        fail(PRISM_BAD_ARG, "prism_jacobi_step_noalloc: n = " + std::to_string(n) + " rows exceeds the fixed scratch of " +
                                std::to_string(PRISM_NOALLOC_MAX_ROWS) + " rows; use prism_solve_csr instead");
    double* scratch = scratchAddress();
    const int rows = (int)n;
    jacobi_csr_kernel<<<ceil_div((int64_t)rows * 32, 256), 256, 0, stream>>>(rows, rowptr, col, values, b, x, scratch); countLaunch();
    PB_LAUNCH("jacobi_csr_kernel");
    copy_kernel<<<ceil_div(rows, 256), 256, 0, stream>>>(rows, scratch, x); countLaunch();
    PB_LAUNCH("copy_kernel");
}

}  // namespace pb
