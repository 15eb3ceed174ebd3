// icb_noalloc.cu — ensemble moments over caller-owned device arrays without
// any device allocation.
//
// Some callers cannot call cudaMalloc: an engine that reserves all device
// memory up front through its own allocator (so a further cudaMalloc fails
// or fragments its pool), or a process that runs under a fixed device-memory
// budget.  icb_moments_noalloc serves them: the caller passes device
// pointers for the inputs and the output, and the per-block partial sums go
// to a fixed file-scope scratch array of this library instead of a buffer
// allocated per call.
//
// Limits and sharing:
//  * the scratch holds kNoAllocMaxItems work items of kNoAllocItemIons ions,
//    so one call accepts at most 4096 * 8192 = 33,554,432 ions (640 KB of
//    scratch, held on every device that loads the library until exit);
//  * every call on a device uses the same scratch: calls that overlap on the
//    GPU (different streams, or other host threads) race and must be
//    serialised by the caller;
//  * the scratch keeps the last call's contents.  Nothing in it has to
//    start at zero: each call writes every partial-sum slot it later reads.
//
// The caller's current device is the same after the call as before it.  The
// scratch array's device address is looked up once per device context (the
// first call on a device, and the first call after that device has been
// reset, since a reset reloads this library's device code at a new
// address); make that first call before any stream capture.
#include <cuda_runtime.h>

#include <mutex>

#include "../../include/icarion_b200.h"
#include "icb_internal.h"

namespace {

constexpr int kNoAllocMaxItems = 4096;
constexpr uint64_t kNoAllocItemIons = 8192;
constexpr int kMaxDevices = 64;

static __device__ __align__(256) double g_noalloc_partials[kNoAllocMaxItems * ICB_N_MOMENTS];

// Device address of the scratch per device, with the unique id of the
// context it was looked up in (0 = not yet looked up).
double* g_scratch_addr[kMaxDevices] = {};
unsigned long long g_scratch_ctx[kMaxDevices] = {};
std::mutex g_scratch_mutex;

// The driver's context queries, reached through the runtime so that the
// library does not link the driver library itself.
using CtxGetCurrentFn = int (*)(void** ctx);
using CtxGetIdFn = int (*)(void* ctx, unsigned long long* id);

// Unique id of the calling thread's current context, or 0 when it cannot be
// had (the caller then looks the address up on every call).
unsigned long long current_context_id() {
    static CtxGetCurrentFn get_current = nullptr;
    static CtxGetIdFn get_id = nullptr;
    static std::once_flag once;
    std::call_once(once, [] {
        void* f = nullptr;
        cudaDriverEntryPointQueryResult q{};
        if (cudaGetDriverEntryPointByVersion("cuCtxGetCurrent", &f, 12000, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            get_current = reinterpret_cast<CtxGetCurrentFn>(f);
        f = nullptr;
        if (cudaGetDriverEntryPointByVersion("cuCtxGetId", &f, 12000, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            get_id = reinterpret_cast<CtxGetIdFn>(f);
    });
    if (!get_current || !get_id) return 0;
    void* ctx = nullptr;
    unsigned long long id = 0;
    if (get_current(&ctx) != 0 || !ctx || get_id(ctx, &id) != 0) return 0;
    return id;
}

// Makes `device` current for the lifetime of the guard and gives the
// caller's current device back on every return path.
class DeviceGuard {
  public:
    explicit DeviceGuard(int device) {
        ok_ = cudaGetDevice(&saved_) == cudaSuccess;
        if (ok_ && saved_ != device) ok_ = cudaSetDevice(device) == cudaSuccess;
        else if (!ok_) saved_ = -1;
        if (!ok_) cudaGetLastError();
    }
    ~DeviceGuard() {
        int cur = -1;
        if (saved_ >= 0 && cudaGetDevice(&cur) == cudaSuccess && cur != saved_) cudaSetDevice(saved_);
    }
    bool ok() const { return ok_; }

  private:
    int saved_ = -1;
    bool ok_ = false;
};

// One block per work item: a fixed-order block reduction of the item's ions
// into partials[item] (slots as ICB_N_MOMENTS).
__global__ void __launch_bounds__(256) k_noalloc_partial(uint64_t n, const double* __restrict__ x,
                                                         const double* __restrict__ y, const double* __restrict__ z,
                                                         const double* __restrict__ vx, const double* __restrict__ vy,
                                                         const double* __restrict__ vz, const double* __restrict__ xr,
                                                         const double* __restrict__ yr, const double* __restrict__ zr,
                                                         const uint8_t* __restrict__ active,
                                                         const double* __restrict__ t_arr,
                                                         const double* __restrict__ t_death,
                                                         double* __restrict__ partials) {
    __shared__ double red[8][ICB_N_MOMENTS];
    const uint64_t begin = static_cast<uint64_t>(blockIdx.x) * kNoAllocItemIons;
    const uint64_t end = begin + kNoAllocItemIons < n ? begin + kNoAllocItemIons : n;
    double acc[ICB_N_MOMENTS];
#pragma unroll
    for (int j = 0; j < ICB_N_MOMENTS; ++j) acc[j] = 0.0;
    for (uint64_t i = begin + threadIdx.x; i < end; i += blockDim.x) {
        if (t_arr && t_arr[i] >= 0.0) acc[11] += 1.0;
        if (!active[i]) {
            if (t_death && t_death[i] >= 0.0) acc[12] += 1.0;
            continue;
        }
        const double px = x[i], py = y[i], pz = z[i];
        const double ux = vx[i], uy = vy[i], uz = vz[i];
        acc[0] += 1.0;
        acc[1] += px; acc[2] += py; acc[3] += pz;
        acc[4] += px * px; acc[5] += py * py; acc[6] += pz * pz;
        acc[7] += ux; acc[8] += uy; acc[9] += uz;
        acc[10] += ux * ux + uy * uy + uz * uz;
        acc[13] += pz * uz;
        const double dx = px - xr[i], dy = py - yr[i], dz = pz - zr[i];
        acc[14] += dx; acc[15] += dy; acc[16] += dz;
        acc[17] += dx * dx; acc[18] += dy * dy; acc[19] += dz * dz;
    }
#pragma unroll
    for (int j = 0; j < ICB_N_MOMENTS; ++j) {
        double v = acc[j];
        for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
        acc[j] = v;
    }
    const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
    if (l == 0) {
#pragma unroll
        for (int j = 0; j < ICB_N_MOMENTS; ++j) red[w][j] = acc[j];
    }
    __syncthreads();
    if (threadIdx.x < ICB_N_MOMENTS) {
        double s = 0.0;
        const int nw = static_cast<int>(blockDim.x >> 5);
        for (int k = 0; k < nw; ++k) s += red[k][threadIdx.x];
        partials[static_cast<size_t>(blockIdx.x) * ICB_N_MOMENTS + threadIdx.x] = s;
    }
}

// Sums the items' partials in item order into out (ICB_N_MOMENTS doubles).
__global__ void k_noalloc_final(const double* __restrict__ partials, int n_items, double* __restrict__ out) {
    if (threadIdx.x >= ICB_N_MOMENTS) return;
    double s = 0.0;
    for (int it = 0; it < n_items; ++it) s += partials[static_cast<size_t>(it) * ICB_N_MOMENTS + threadIdx.x];
    out[threadIdx.x] = s;
}

}  // namespace

extern "C" int icb_moments_noalloc(int device, uint64_t n, const double* x, const double* y, const double* z,
                                   const double* vx, const double* vy, const double* vz,
                                   const double* x_ref, const double* y_ref, const double* z_ref,
                                   const uint8_t* active, const double* arrival_time_s,
                                   const double* death_time_s, double* out, void* cuda_stream) {
    using icb::set_error;
    if (device < 0 || device >= kMaxDevices) return set_error(ICB_ERR_INVALID_ARGUMENT, "device ordinal out of range");
    if (n == 0 || !x || !y || !z || !vx || !vy || !vz || !x_ref || !y_ref || !z_ref || !active || !out)
        return set_error(ICB_ERR_INVALID_ARGUMENT, "icb_moments_noalloc: n must be > 0 and the arrays non-NULL");
    const uint64_t items = (n + kNoAllocItemIons - 1) / kNoAllocItemIons;
    if (items > static_cast<uint64_t>(kNoAllocMaxItems))
        return set_error(ICB_ERR_INVALID_ARGUMENT,
                         "icb_moments_noalloc: at most 33554432 ions (the fixed 640 KB scratch holds 4096 partial sums)");
    DeviceGuard guard(device);
    if (!guard.ok()) return set_error(ICB_ERR_NO_DEVICE, "cudaSetDevice failed");
    double* scratch = nullptr;
    {
        std::lock_guard<std::mutex> lock(g_scratch_mutex);
        const unsigned long long ctx = current_context_id();
        if (!g_scratch_addr[device] || ctx == 0 || ctx != g_scratch_ctx[device]) {
            // First call in this device's context: resolve the scratch
            // array's device address with the device current.
            void* ptr = nullptr;
            if (cudaGetSymbolAddress(&ptr, g_noalloc_partials) != cudaSuccess || !ptr) {
                g_scratch_addr[device] = nullptr;
                return set_error(ICB_ERR_CUDA, "cudaGetSymbolAddress of the moments scratch failed");
            }
            g_scratch_addr[device] = static_cast<double*>(ptr);
            g_scratch_ctx[device] = ctx;
        }
        scratch = g_scratch_addr[device];
    }
    cudaStream_t s = static_cast<cudaStream_t>(cuda_stream);
    k_noalloc_partial<<<static_cast<unsigned>(items), 256, 0, s>>>(n, x, y, z, vx, vy, vz, x_ref, y_ref, z_ref,
                                                                   active, arrival_time_s, death_time_s, scratch);
    if (cudaGetLastError() != cudaSuccess) return set_error(ICB_ERR_CUDA, "moments partial kernel launch failed");
    k_noalloc_final<<<1, 32, 0, s>>>(scratch, static_cast<int>(items), out);
    if (cudaGetLastError() != cudaSuccess) return set_error(ICB_ERR_CUDA, "moments final kernel launch failed");
    return ICB_OK;
}
