// acfd_cfl_noalloc: the CFL wave-speed maximum (solve.c:132-151) for callers
// that cannot allocate device memory.
//
// Some hosts must not call cudaMalloc/cudaFree from the time loop: programs
// whose device memory is owned by a pool allocator (PyTorch's caching
// allocator, RMM) that has to see every allocation, and long-running solvers
// with a memory budget fixed at start-up, where a late cudaMalloc can fail and
// cudaFree synchronizes the whole device.  This variant takes the state and
// the output from the caller and keeps its only scratch -- one partial maximum
// per block and direction plus one non-finite flag per block -- in a
// file-scope __device__ array of fixed size, so the call allocates nothing.
//
// Compiled with --fmad=false: the result is bitwise that of acfd_cfl.
#include <cuda.h>
#include <cudaTypedefs.h>

#include <mutex>

#include "acfd_internal.cuh"

namespace acfd {
namespace {

// scratch: per block 3 partial maxima and 1 non-finite flag; 4096 blocks x 4
// doubles = 128 KiB held on every device that loads the library, until the
// process exits
constexpr int kNoAllocMaxBlocks = 4096;
constexpr int kNoAllocThreads = 256;
constexpr long long kNodesPerBlockMax = 8192;  // the size limit: 4096 x 8192 nodes
constexpr long long kNodesPerBlock = 1024;     // launch size: several blocks per SM at 2 M nodes
constexpr int kMaxDevices = 64;

__device__ __align__(256) double g_cfl_scratch[4 * kNoAllocMaxBlocks];

std::mutex g_setup_mutex;
// the scratch address of each device, with the context it was looked up in:
// a device reset or a new primary context loads the module again at another
// address, so the address is looked up again when the context changes
double *g_scratch_addr[kMaxDevices] = {nullptr};
CUcontext g_scratch_ctx[kMaxDevices] = {nullptr};

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
    bool bad = false;  // a fluid node whose wave speed is not finite
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
        const double v0 = fabs(u) + c, v1 = fabs(v) + c, v2 = fabs(w) + c;
        m0 = wave_max(m0, v0);
        m1 = wave_max(m1, v1);
        m2 = wave_max(m2, v2);
        bad = bad || !isfinite(v0 + v1 + v2);
    }
    for (int o = 16; o > 0; o >>= 1) {
        m0 = wave_max(m0, __shfl_xor_sync(0xffffffffu, m0, o));
        m1 = wave_max(m1, __shfl_xor_sync(0xffffffffu, m1, o));
        m2 = wave_max(m2, __shfl_xor_sync(0xffffffffu, m2, o));
    }
    const int any_bad = __syncthreads_or(bad ? 1 : 0);
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
    } else if (threadIdx.x == 3) {
        part[3 * kNoAllocMaxBlocks + blockIdx.x] = any_bad ? 1.0 : 0.0;
    }
}

// every slot read here was written by cfl_noalloc_partial earlier in the same
// call on the same stream, so the scratch needs no clearing between calls.
// When any block met a fluid node with a non-finite wave speed the three
// outputs are NaN: the call returns before the kernels run, so the state's
// failure travels in the values themselves.
__global__ void cfl_noalloc_final(const double *__restrict__ part, int nblocks, double *__restrict__ out)
{
    __shared__ double sm[3][32];
    __shared__ int any_bad;
    if (threadIdx.x == 0) {
        any_bad = 0;
    }
    __syncthreads();
    const int s = threadIdx.x >> 5, lane = threadIdx.x & 31;
    if (s < 3) {
        double m = 0.0;
        for (int b = lane; b < nblocks; b += 32) {
            m = wave_max(m, part[3 * b + s]);
        }
        sm[s][lane] = m;
    } else {
        int bad = 0;
        for (int b = lane; b < nblocks; b += 32) {
            bad |= part[3 * kNoAllocMaxBlocks + b] != 0.0;
        }
        if (__any_sync(0xffffffffu, bad) && lane == 0) {
            any_bad = 1;
        }
    }
    __syncthreads();
    if (threadIdx.x < 3) {
        double m = 0.0;
        for (int q = 0; q < 32; ++q) {
            m = wave_max(m, sm[threadIdx.x][q]);
        }
        out[threadIdx.x] = any_bad ? __longlong_as_double(0x7ff8000000000000LL) : m;
    }
}

PFN_cuCtxGetCurrent_v4000 ctx_getter()
{
    static PFN_cuCtxGetCurrent_v4000 fn = nullptr;
    if (!fn) {
        void *p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &p, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess) {
            fn = reinterpret_cast<PFN_cuCtxGetCurrent_v4000>(p);
        }
    }
    return fn;
}

// per-device set-up: the device address of the scratch array (host code may
// not use the symbol itself as a pointer), looked up once per device and
// context
int scratch_for_current_device(double **out)
{
    int dev = 0;
    ACFD_CUDA(cudaGetDevice(&dev));
    if (dev < 0 || dev >= kMaxDevices) {
        set_error("acfd_cfl_noalloc: device ordinal %d beyond %d", dev, kMaxDevices);
        return ACFD_ERR_ARG;
    }
    std::lock_guard<std::mutex> lock(g_setup_mutex);
    PFN_cuCtxGetCurrent_v4000 get_ctx = ctx_getter();
    CUcontext ctx = nullptr;
    if (!get_ctx || get_ctx(&ctx) != CUDA_SUCCESS) {
        set_error("acfd_cfl_noalloc: cuCtxGetCurrent not available from the driver");
        return ACFD_ERR_CUDA;
    }
    if (!g_scratch_addr[dev] || g_scratch_ctx[dev] != ctx) {
        void *p = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&p, g_cfl_scratch);
        if (e != cudaSuccess) {
            return cuda_status(e, "cudaGetSymbolAddress(g_cfl_scratch)");
        }
        if (!ctx && get_ctx(&ctx) != CUDA_SUCCESS) {
            ctx = nullptr;  // the runtime made the primary context current just now
        }
        g_scratch_addr[dev] = static_cast<double *>(p);
        g_scratch_ctx[dev] = ctx;
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
        if (g.lo[s] < 0 || g.hi[s] > g.n[s] || g.hi[s] < g.lo[s]) {
            set_error("acfd_cfl_noalloc: PIN range [%d, %d) not inside the node array [0, %d) on axis %d",
                      g.lo[s], g.hi[s], g.n[s], s);
            return ACFD_ERR_ARG;
        }
    }
    g.pitch = pitch;
    g.nn = (long long)pitch * g.n[1] * g.n[2];
    const long long pin = (long long)(g.hi[0] - g.lo[0]) * (g.hi[1] - g.lo[1]) * (g.hi[2] - g.lo[2]);
    const long long max_pin = (long long)kNoAllocMaxBlocks * kNodesPerBlockMax;
    if (pin > max_pin) {
        set_error("acfd_cfl_noalloc: %lld computed nodes exceed the fixed scratch limit of %lld "
                  "(%d blocks x %lld nodes); use acfd_cfl", pin, max_pin, kNoAllocMaxBlocks, kNodesPerBlockMax);
        return ACFD_ERR_ARG;
    }
    double *scratch = nullptr;
    const int st = scratch_for_current_device(&scratch);
    if (st != ACFD_OK) {
        return st;
    }
    long long blocks = (pin + kNodesPerBlock - 1) / kNodesPerBlock;
    if (blocks < 1) blocks = 1;
    if (blocks > kNoAllocMaxBlocks) blocks = kNoAllocMaxBlocks;  // the grid-stride loop covers the rest
    cudaStream_t cs = static_cast<cudaStream_t>(stream);
    cfl_noalloc_partial<<<(unsigned)blocks, kNoAllocThreads, 0, cs>>>(g, model->gamma, model->gasR, U_to, did,
                                                                       scratch);
    cfl_noalloc_final<<<1, 128, 0, cs>>>(scratch, (int)blocks, vmax_dev);
    cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? ACFD_OK : cuda_status(e, "acfd_cfl_noalloc launch");
}
