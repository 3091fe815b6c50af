// acfd_cfl_noalloc: the CFL wave-speed maximum (solve.c:132-151) for callers
// that cannot allocate device memory.
//
// Some hosts must not call cudaMalloc/cudaFree from the time loop: programs
// whose device memory is owned by a pool allocator (PyTorch's caching
// allocator, RMM) that has to see every allocation, and long-running solvers
// with a memory budget fixed at start-up, where a late cudaMalloc can fail and
// cudaFree synchronizes the whole device.  This variant takes the state and
// the output from the caller and keeps its only scratch -- one partial maximum
// per block -- in a file-scope __device__ array of fixed size, so the call
// allocates nothing.
//
// Compiled with --fmad=false: the result is bitwise that of acfd_cfl.
#include <mutex>

#include "acfd_internal.cuh"

namespace acfd {
namespace {

// scratch: 3 partial maxima per block; 4096 blocks x 3 doubles = 96 KiB held
// on every device that loads the library, until the process exits
constexpr int kNoAllocMaxBlocks = 4096;
constexpr int kNoAllocThreads = 256;
constexpr long long kNodesPerBlock = 8192;  // PIN nodes one block reduces
constexpr int kMaxDevices = 64;

__device__ __align__(256) double g_cfl_scratch[3 * kNoAllocMaxBlocks];

std::mutex g_setup_mutex;
double *g_scratch_addr[kMaxDevices] = {nullptr};

__device__ __forceinline__ double wave_max(double a, double b)
{
    return (a < b) ? b : a;  // a NaN never replaces the running maximum
}

__global__ void __launch_bounds__(kNoAllocThreads)
cfl_noalloc_partial(Grid g, double gamma, double gasR, const double *__restrict__ U,
                    const int *__restrict__ did, double *__restrict__ part)
{
    const int Lx = g.hi[0] - g.lo[0], Ly = g.hi[1] - g.lo[1], Lz = g.hi[2] - g.lo[2];
    const long long total = (long long)Lx * Ly * Lz;
    double m0 = 0.0, m1 = 0.0, m2 = 0.0;
    for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < total;
         t += (long long)gridDim.x * blockDim.x) {
        const int i = g.lo[0] + (int)(t % Lx);
        const long long rest = t / Lx;
        const int j = g.lo[1] + (int)(rest % Ly);
        const int k = g.lo[2] + (int)(rest / Ly);
        const long long id = ((long long)k * g.n[1] + j) * g.pitch + i;
        if (did[id] != 0) {
            continue;
        }
        // MapPrimitive (cfd_commons.c:296-305), then |u_s| + sqrt(gamma*gasR*T)
        const double r = U[id];
        const double mx = U[g.nn + id], my = U[2 * g.nn + id], mz = U[3 * g.nn + id];
        const double e = U[4 * g.nn + id];
        const double u = mx / r, v = my / r, w = mz / r;
        const double p = (e - 0.5 * (mx * mx + my * my + mz * mz) / r) * (gamma - 1.0);
        const double T = p / (r * gasR);
        const double c = sqrt(gamma * gasR * T);
        m0 = wave_max(m0, fabs(u) + c);
        m1 = wave_max(m1, fabs(v) + c);
        m2 = wave_max(m2, fabs(w) + c);
    }
    for (int o = 16; o > 0; o >>= 1) {
        m0 = wave_max(m0, __shfl_xor_sync(0xffffffffu, m0, o));
        m1 = wave_max(m1, __shfl_xor_sync(0xffffffffu, m1, o));
        m2 = wave_max(m2, __shfl_xor_sync(0xffffffffu, m2, o));
    }
    __shared__ double sm[3][kNoAllocThreads / 32];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    if (lane == 0) {
        sm[0][warp] = m0;
        sm[1][warp] = m1;
        sm[2][warp] = m2;
    }
    __syncthreads();
    if (threadIdx.x < 3) {
        double m = 0.0;
        for (int q = 0; q < kNoAllocThreads / 32; ++q) {
            m = wave_max(m, sm[threadIdx.x][q]);
        }
        part[3 * blockIdx.x + threadIdx.x] = m;
    }
}

// every slot read here was written by cfl_noalloc_partial earlier in the same
// call on the same stream, so the scratch needs no clearing between calls
__global__ void cfl_noalloc_final(const double *__restrict__ part, int nblocks, double *__restrict__ out)
{
    __shared__ double sm[3][32];
    const int s = threadIdx.x >> 5, lane = threadIdx.x & 31;
    if (s < 3) {
        double m = 0.0;
        for (int b = lane; b < nblocks; b += 32) {
            m = wave_max(m, part[3 * b + s]);
        }
        sm[s][lane] = m;
    }
    __syncthreads();
    if (threadIdx.x < 3) {
        double m = 0.0;
        for (int q = 0; q < 32; ++q) {
            m = wave_max(m, sm[threadIdx.x][q]);
        }
        out[threadIdx.x] = m;
    }
}

// per-device set-up: the device address of the scratch array (host code may
// not use the symbol itself as a pointer)
int scratch_for_current_device(double **out)
{
    int dev = 0;
    ACFD_CUDA(cudaGetDevice(&dev));
    if (dev < 0 || dev >= kMaxDevices) {
        set_error("acfd_cfl_noalloc: device ordinal %d beyond %d", dev, kMaxDevices);
        return ACFD_ERR_ARG;
    }
    std::lock_guard<std::mutex> lock(g_setup_mutex);
    if (!g_scratch_addr[dev]) {
        void *p = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&p, g_cfl_scratch);
        if (e != cudaSuccess) {
            return cuda_status(e, "cudaGetSymbolAddress(g_cfl_scratch)");
        }
        g_scratch_addr[dev] = static_cast<double *>(p);
    }
    *out = g_scratch_addr[dev];
    return ACFD_OK;
}

}  // namespace
}  // namespace acfd

extern "C" int acfd_cfl_noalloc(const acfd_partition_t *part, const acfd_model_t *model, const double *U_to,
                                const int *did, int pitch, double *vmax_dev, void *stream)
{
    using namespace acfd;
    if (!part || !model || !U_to || !did || !vmax_dev) {
        set_error("acfd_cfl_noalloc: null argument");
        return ACFD_ERR_ARG;
    }
    if (pitch < part->n[0]) {
        set_error("acfd_cfl_noalloc: pitch %d smaller than n[X] = %d", pitch, part->n[0]);
        return ACFD_ERR_ARG;
    }
    Grid g;
    for (int s = 0; s < 3; ++s) {
        g.n[s] = part->n[s];
        g.lo[s] = part->ns[0][s][0];
        g.hi[s] = part->ns[0][s][1];
        g.dd[s] = part->dd[s];
        if (g.lo[s] < 0 || g.hi[s] > g.n[s]) {
            set_error("acfd_cfl_noalloc: PIN range outside the node array on axis %d", s);
            return ACFD_ERR_ARG;
        }
    }
    g.pitch = pitch;
    g.nn = (long long)pitch * g.n[1] * g.n[2];
    const long long pin = (long long)(g.hi[0] - g.lo[0]) * (g.hi[1] - g.lo[1]) * (g.hi[2] - g.lo[2]);
    const long long max_pin = (long long)kNoAllocMaxBlocks * kNodesPerBlock;
    if (pin > max_pin) {
        set_error("acfd_cfl_noalloc: %lld computed nodes exceed the fixed scratch limit of %lld "
                  "(%d blocks x %lld nodes); use acfd_cfl", pin, max_pin, kNoAllocMaxBlocks, kNodesPerBlock);
        return ACFD_ERR_ARG;
    }
    double *scratch = nullptr;
    const int st = scratch_for_current_device(&scratch);
    if (st != ACFD_OK) {
        return st;
    }
    long long blocks = (pin + kNodesPerBlock - 1) / kNodesPerBlock;
    if (blocks < 1) blocks = 1;
    cudaStream_t cs = static_cast<cudaStream_t>(stream);
    cfl_noalloc_partial<<<(unsigned)blocks, kNoAllocThreads, 0, cs>>>(g, model->gamma, model->gasR, U_to, did,
                                                                       scratch);
    cfl_noalloc_final<<<1, 96, 0, cs>>>(scratch, (int)blocks, vmax_dev);
    cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? ACFD_OK : cuda_status(e, "acfd_cfl_noalloc launch");
}
