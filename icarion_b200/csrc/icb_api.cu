// icb_api.cu — the C ABI (include/icarion_b200.h): handle lifetime, device
// resident SoA ion state, launch sequencing, the device engine clock and the
// deterministic per-ensemble moment reduction.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <memory>
#include <string>
#include <vector>

#include "../../include/icarion_b200.h"
#include "icb_internal.h"
#include "icb_params.h"
#include "icb_rng.cuh"

using namespace icb;

// ---------------------------------------------------------------------------
// errors
// ---------------------------------------------------------------------------
namespace {
thread_local std::string g_last_error;

int fail(int code, const char* fmt, ...) {
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    std::vsnprintf(buf, sizeof(buf), fmt, ap);
    va_end(ap);
    g_last_error = buf;
    return code;
}

#define ICB_CUDA(call)                                                                   \
    do {                                                                                 \
        cudaError_t err_ = (call);                                                       \
        if (err_ != cudaSuccess) {                                                       \
            return fail(err_ == cudaErrorMemoryAllocation ? ICB_ERR_OUT_OF_MEMORY        \
                                                          : ICB_ERR_CUDA,                \
                        "%s failed: %s (%s:%d)", #call, cudaGetErrorString(err_),        \
                        __FILE__, __LINE__);                                             \
        }                                                                                \
    } while (0)

constexpr double kGeomEps = 1e-12;          // CylindricalGeometry.h:245
constexpr double kMinVoltage = 1e-12;       // AnalyticalFieldModel voltage threshold
constexpr double kBoltzmann = 1.380649e-23; // utils/constants.h:15
constexpr double kEps0 = 8.854187817e-12;   // utils/constants.h:19
constexpr double kMeanChi3 = 1.5957691216057308;  // E|N(0,I3)| = 2 sqrt(2/pi)
constexpr int kMomItemIons = 8192;

template <class T>
struct DevBuf {
    T* p = nullptr;
    size_t n = 0;
    ~DevBuf() { if (p) cudaFree(p); }
    cudaError_t alloc(size_t count) {
        if (p) { cudaFree(p); p = nullptr; n = 0; }
        if (count == 0) return cudaSuccess;
        cudaError_t e = cudaMalloc(reinterpret_cast<void**>(&p), count * sizeof(T));
        if (e == cudaSuccess) n = count;
        return e;
    }
};

}  // namespace

int icb::set_error(int code, const char* msg) {
    g_last_error = msg;
    return code;
}

// ---------------------------------------------------------------------------
// auxiliary kernels
// ---------------------------------------------------------------------------
namespace {

// Initial collision clocks from u = uniform of Philox(id, 0, 3, 0).x:
// per-step clock S = 1, U = u; skip clock tau = -ln u, restart pending.
template <class R>
__global__ void k_clock_init(R* S, R* U, uint32_t* nxt, uint32_t* start, uint64_t n, uint64_t first_id,
                             uint64_t seed, int skip) {
    const uint64_t i = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const U4 r = philox4x32_10(static_cast<uint32_t>(first_id + i), 0u, 3u, 0u,
                               static_cast<uint32_t>(seed), static_cast<uint32_t>(seed >> 32));
    R u;
    if constexpr (sizeof(R) == 8) u = unit_d(r.x);
    else u = 2.0f - __uint_as_float(0x3f800000u | (r.x >> 9));
    if (skip) {
        S[i] = -log(u);
        U[i] = R(0);
        nxt[i] = 0xFFFFFFFFu;
        start[i] = 0u;
    } else {
        S[i] = R(1);
        U[i] = u;
    }
}

// Device engine clock: step += K and t_e += dt_e, K times (accumulated like
// the engine's per-step t += dt, SimulationEngineLifecycle.cpp:162).
__global__ void k_clock_advance(unsigned long long* step, double* t, const double* dt, int n_ens, uint32_t K) {
    const int e = static_cast<int>(blockIdx.x * blockDim.x + threadIdx.x);
    if (e == 0) *step += K;
    if (e >= n_ens) return;
    double te = t[e];
    const double d = dt[e];
    for (uint32_t k = 0; k < K; ++k) te = te + d;
    t[e] = te;
}

// Upload conversion: staged doubles -> working precision.
__global__ void k_to_float(const double* __restrict__ src, float* __restrict__ dst, uint64_t n) {
    const uint64_t i = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i < n) dst[i] = static_cast<float>(src[i]);
}
__global__ void k_to_hilo(const double* __restrict__ src, float* __restrict__ hi, float* __restrict__ lo, uint64_t n) {
    const uint64_t i = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i < n) {
        const float h = static_cast<float>(src[i]);
        hi[i] = h;
        lo[i] = static_cast<float>(src[i] - static_cast<double>(h));
    }
}
__global__ void k_from_float(const float* __restrict__ src, double* __restrict__ dst, uint64_t n) {
    const uint64_t i = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i < n) dst[i] = static_cast<double>(src[i]);
}
__global__ void k_from_hilo(const float* __restrict__ hi, const float* __restrict__ lo, double* __restrict__ dst, uint64_t n) {
    const uint64_t i = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i < n) dst[i] = static_cast<double>(hi[i]) + static_cast<double>(lo[i]);
}
__global__ void k_flags_in(const uint8_t* __restrict__ active, const double* __restrict__ birth, uint8_t* __restrict__ flags,
                           double* __restrict__ t_death, double* __restrict__ t_arr, uint64_t n) {
    const uint64_t i = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const bool born = birth == nullptr || birth[i] <= 0.0;
    uint8_t f = 0;
    if (born) f |= kFlagBorn;
    if (born && active[i]) f |= kFlagActive;
    flags[i] = f;
    t_death[i] = -1.0;
    t_arr[i] = -1.0;
}
__global__ void k_flags_update(const uint8_t* __restrict__ active, uint8_t* __restrict__ flags, uint64_t n) {
    const uint64_t i = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= n) return;
    uint8_t f = flags[i];
    if ((f & kFlagBorn) != 0) f = active[i] ? static_cast<uint8_t>(f | kFlagActive) : static_cast<uint8_t>(f & ~kFlagActive);
    flags[i] = f;
}
__global__ void k_flags_out(const uint8_t* __restrict__ flags, uint8_t* __restrict__ active, uint64_t n) {
    const uint64_t i = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i < n) active[i] = (flags[i] & kFlagActive) ? 1 : 0;
}
// One ion chunk of the overlapped host path, in one launch each way: the
// staged double velocities (three arrays `stride` apart) to float when vx is
// given, and the host activity bytes into the flags (k_to_float x 3 +
// k_flags_update); and back (k_from_float x 3 + k_flags_out).
__global__ void k_chunk_in(const double* __restrict__ stage, uint64_t stride, float* __restrict__ vx,
                           float* __restrict__ vy, float* __restrict__ vz, const uint8_t* __restrict__ active,
                           uint8_t* __restrict__ flags, uint64_t n) {
    const uint64_t i = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= n) return;
    if (vx) {
        vx[i] = static_cast<float>(stage[i]);
        vy[i] = static_cast<float>(stage[stride + i]);
        vz[i] = static_cast<float>(stage[2 * stride + i]);
    }
    uint8_t f = flags[i];
    if ((f & kFlagBorn) != 0) f = active[i] ? static_cast<uint8_t>(f | kFlagActive) : static_cast<uint8_t>(f & ~kFlagActive);
    flags[i] = f;
}
__global__ void k_chunk_out(const float* __restrict__ vx, const float* __restrict__ vy, const float* __restrict__ vz,
                            double* __restrict__ stage, uint64_t stride, const uint8_t* __restrict__ flags,
                            uint8_t* __restrict__ active, uint64_t n) {
    const uint64_t i = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= n) return;
    if (vx) {
        stage[i] = static_cast<double>(vx[i]);
        stage[stride + i] = static_cast<double>(vy[i]);
        stage[2 * stride + i] = static_cast<double>(vz[i]);
    }
    active[i] = (flags[i] & kFlagActive) ? 1 : 0;
}

// Moments: one block per work item (a slice of one ensemble's ions), a
// fixed-order block reduction into partials[item], then one block per
// ensemble sums its items in order.  Deterministic for a given item split.
struct MomItem { uint64_t begin, end; };

template <class R, bool HILO>
__global__ void __launch_bounds__(256) k_moments_partial(const MomItem* __restrict__ items,
                                                         const double* __restrict__ x, const double* __restrict__ y, const double* __restrict__ z,
                                                         const float* __restrict__ xh, const float* __restrict__ xl,
                                                         const float* __restrict__ yh, const float* __restrict__ yl,
                                                         const float* __restrict__ zh, const float* __restrict__ zl,
                                                         const R* __restrict__ vx, const R* __restrict__ vy, const R* __restrict__ vz,
                                                         const double* __restrict__ xr, const double* __restrict__ yr, const double* __restrict__ zr,
                                                         const uint8_t* __restrict__ flags, const double* __restrict__ t_death,
                                                         const double* __restrict__ t_arr, double* __restrict__ partials) {
    __shared__ double red[8][ICB_N_MOMENTS];
    const MomItem it = items[blockIdx.x];
    double acc[ICB_N_MOMENTS];
#pragma unroll
    for (int j = 0; j < ICB_N_MOMENTS; ++j) acc[j] = 0.0;
    for (uint64_t i = it.begin + threadIdx.x; i < it.end; i += blockDim.x) {
        const uint8_t f = flags[i];
        if (t_arr[i] >= 0.0) acc[11] += 1.0;
        if (!(f & kFlagActive)) {
            if (t_death[i] >= 0.0) acc[12] += 1.0;
            continue;
        }
        double px, py, pz;
        if constexpr (HILO) {
            px = static_cast<double>(xh[i]) + static_cast<double>(xl[i]);
            py = static_cast<double>(yh[i]) + static_cast<double>(yl[i]);
            pz = static_cast<double>(zh[i]) + static_cast<double>(zl[i]);
        } else {
            px = x[i]; py = y[i]; pz = z[i];
        }
        const double ux = static_cast<double>(vx[i]), uy = static_cast<double>(vy[i]), uz = static_cast<double>(vz[i]);
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

__global__ void k_moments_final(const double* __restrict__ partials, const int* __restrict__ item_off,
                                int n_ens, double* __restrict__ out) {
    const int e = blockIdx.x;
    if (e >= n_ens || threadIdx.x >= ICB_N_MOMENTS) return;
    double s = 0.0;
    for (int it = item_off[e]; it < item_off[e + 1]; ++it) s += partials[static_cast<size_t>(it) * ICB_N_MOMENTS + threadIdx.x];
    out[static_cast<size_t>(e) * ICB_N_MOMENTS + threadIdx.x] = s;
}

}  // namespace

// ---------------------------------------------------------------------------
// handle
// ---------------------------------------------------------------------------
struct icb_handle {
    icb_config cfg{};
    std::vector<icb_ensemble_params> ens;
    std::vector<EnsConst> ens_const;
    int field_kind = kFieldUniform;
    bool magnetic = false;
    int coll = kCollNone;
    int block = 128;
    uint32_t K = 1000;
    uint32_t pend = 0;      // 0 = precision default (set at create)
    uint32_t spv = 8;       // collision-free steps between warp votes
    bool shape_tuned = false;  // block / pend / spv chosen by icb_autotune
    // per-step mode: the last launch finalized every ion and nothing wrote
    // the state since, so every live ion is inside its domain (the next
    // step's prepare has nothing to remove)
    bool prep_ok = false;
    // space charge: the field bound is automatic (4 x the largest field);
    // it was taken again with the peers' ions; the peers last set
    bool sc_bound_auto = false, sc_peers_bounded = false;
    const void* sc_peer_ptr = nullptr;
    uint64_t sc_peer_n = 0, sc_peer_skip_b = 0, sc_peer_skip_n = 0;
    std::vector<double> sp_m, sp_q;   // per ensemble: shared ion mass / charge (0 = per ion)
    cudaStream_t own_stream = nullptr;
    cudaStream_t stream = nullptr;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    std::vector<cudaEvent_t> kev;      // per-launch events of the step kernel
    uint64_t launches = 0;             // kernels launched by the current call
    uint64_t host_step = 0;            // host mirror of the engine step index

    uint64_t n = 0;
    uint64_t first_id = 0;
    std::vector<uint64_t> ens_off;

    DevBuf<double> x, y, z;
    DevBuf<double> xr, yr, zr;   // displacement reference positions
    DevBuf<float> xh, xl, yh, yl, zh, zl;
    DevBuf<double> vxd, vyd, vzd;
    DevBuf<float> vxf, vyf, vzf;
    DevBuf<double> Sd, Ud;
    DevBuf<float> Sf, Uf;
    DevBuf<uint32_t> clk_next, clk_start;   // skip clock (Boris + collisions)
    DevBuf<double> mass, charge, t_death, t_arr, birth, zprev;
    DevBuf<uint8_t> flags, active_stage;
    DevBuf<double> stage;
    DevBuf<unsigned long long> counters, step_dev;
    DevBuf<double> t_dev, dt_dev;
    DevBuf<MomItem> mom_items;
    DevBuf<int> mom_item_off;
    DevBuf<double> mom_partials, mom_out;
    int n_mom_items = 0;
    bool has_birth = false;

    bool fp64() const { return cfg.precision == ICB_PREC_FP64; }
    bool skip_clock() const { return coll != kCollNone && cfg.integrator == ICB_INTEGRATOR_BORIS; }
    bool hilo() const { return cfg.precision == ICB_PREC_MIXED_HILO; }
    void* vx() const { return fp64() ? static_cast<void*>(vxd.p) : static_cast<void*>(vxf.p); }
    void* vy() const { return fp64() ? static_cast<void*>(vyd.p) : static_cast<void*>(vyf.p); }
    void* vz() const { return fp64() ? static_cast<void*>(vzd.p) : static_cast<void*>(vzf.p); }
    // CUDA graph of one icb_advance(graph_steps) launch sequence; rebuilt when
    // anything baked into it changes (state arrays, stream, launch shape).
    cudaGraphExec_t graph = nullptr;
    uint64_t graph_steps = 0;
    uint64_t graph_gen = 0;
    uint64_t graph_launches = 0;
    uint64_t gen = 1;                  // bumped whenever the graph goes stale
    // interaction-potential collisions: cos(chi) table and learned model
    DevBuf<float> ipm_tab;
    int ipm_nE = 0, ipm_nb = 0;
    double ipm_lnEmin = 0.0, ipm_inv_dlnE = 0.0, ipm_bmax = 0.0, ipm_Emin = 0.0, ipm_Emax = 0.0;
    double ipm_net_lnEmin = 0.0, ipm_net_scale = 0.0;   // x0 = (ln E - lnEmin) scale - 1
    IpmPotential ipm_pot{};
    const GLNodes* ipm_gl = nullptr;
    DevBuf<uint32_t> mlp_w2;
    DevBuf<float> mlp_f;
    DevBuf<MixConst> mix;              // HSS gas mixtures, per ensemble
    // time-dependent fields: waveforms per (ensemble, channel), TIMS axial
    // fields, and the device table built from them
    std::vector<icb_waveform> waves;   // n_ens * ICB_N_CHANNELS
    std::vector<uint8_t> wave_set;
    std::vector<icb_tims_field> tims;
    std::vector<uint8_t> tims_set;
    DevBuf<TimeField> tfield;
    DevBuf<double> tf_tab;             // per-step field scalars, one launch chunk at a time
    bool any_tf = false;
    int base_field_kind = kFieldUniform;
    // EHSS geometry: host copies per ensemble and the device arrays
    std::vector<std::vector<double4>> ehss_host;
    std::vector<double> ehss_rgas_host;
    DevBuf<double4> ehss_atoms;
    DevBuf<int32_t> ehss_off;
    DevBuf<double> ehss_rgas;
    bool mlp_ready = false;
    // host fast path: copy and copy-back streams, per-chunk compute streams
    // and events, velocity staging (3n)
    cudaStream_t copy_stream = nullptr, copy_back_stream = nullptr;
    std::vector<cudaStream_t> chunk_streams;
    std::vector<cudaEvent_t> hev;
    DevBuf<double> hstage;
    // space charge (solved before every step when configured)
    SpaceChargeSolver* sc = nullptr;
    double sc_emax_base = 0.0;         // ensemble 0's field bound without space charge
    std::vector<cudaEvent_t> sc_ev;    // per-solve events (first 64 solves of a call)
    size_t sc_timed = 0;
    void drop_graph() {
        if (graph) cudaGraphExecDestroy(graph);
        graph = nullptr;
        graph_steps = 0;
    }

    ~icb_handle() {
        drop_graph();
        if (sc) sc_destroy(sc);
        for (cudaEvent_t e : sc_ev) cudaEventDestroy(e);
        for (cudaEvent_t e : hev) cudaEventDestroy(e);
        if (copy_stream) cudaStreamDestroy(copy_stream);
        if (copy_back_stream) cudaStreamDestroy(copy_back_stream);
        for (cudaStream_t cst : chunk_streams) cudaStreamDestroy(cst);
        for (cudaEvent_t e : kev) cudaEventDestroy(e);
        if (ev0) cudaEventDestroy(ev0);
        if (ev1) cudaEventDestroy(ev1);
        if (own_stream) cudaStreamDestroy(own_stream);
    }
};

namespace {

int check_handle(icb_handle* h) {
    if (!h) return fail(ICB_ERR_INVALID_ARGUMENT, "null handle");
    cudaError_t e = cudaSetDevice(h->cfg.device);
    if (e != cudaSuccess) return fail(ICB_ERR_CUDA, "cudaSetDevice(%d): %s", h->cfg.device, cudaGetErrorString(e));
    return ICB_OK;
}

// Upper bound of |E| over the cylinder for E = E0 + G .* (x - c) plus the
// RF quadrupole term: |E0| + |G .* max|x - c|| + 2 (|U0| + |V|) r_axis / r0^2.
// The CPU oracle evaluates the same expression (orc_field_bound).
double field_bound(const EnsConst& C, const icb_ensemble_params& P) {
    const double Rp = P.radius_m + kGeomEps;
    double e = std::sqrt(C.E0[0] * C.E0[0] + C.E0[1] * C.E0[1] + C.E0[2] * C.E0[2]);
    const double ex = std::fabs(C.ox - C.c[0]) + Rp;
    const double ey = std::fabs(C.oy - C.c[1]) + Rp;
    const double ez = std::fmax(std::fabs(C.oz - C.c[2]), std::fabs(C.oz + C.zmax_local - C.c[2]));
    const double gx = C.G[0] * ex, gy = C.G[1] * ey, gz = C.G[2] * ez;
    e = e + std::sqrt(gx * gx + gy * gy + gz * gz);
    if (C.rf) {
        const double dx = C.ox - C.c[0], dy = C.oy - C.c[1];
        const double raxis = std::sqrt(dx * dx + dy * dy) + Rp;
        e = e + 2.0 * (std::fabs(C.rf_U0) + std::fabs(C.rf_V)) * raxis / C.r0sq;
    }
    if (C.ac) e = e + (std::fabs(C.ac_amp[0]) + std::fabs(C.ac_amp[1]));
    return e;
}

// Largest |value| a waveform takes at any time (infinite when unbounded).
double wave_bound(const icb_waveform& w) {
    const double* p = w.p;
    switch (w.type) {
        case ICB_WAVE_CONSTANT: return std::fabs(p[0]);
        case ICB_WAVE_LINEAR: return std::fmax(std::fabs(p[0]), std::fabs(p[1]));
        case ICB_WAVE_QUADRATIC: {
            auto q = [&](double t) { return std::fabs(p[0] + p[1] * t + p[2] * t * t); };
            double b = std::fmax(std::fabs(p[0]), std::fmax(q(p[3]), q(p[4])));
            if (p[2] != 0.0) {
                const double tv = -p[1] / (2.0 * p[2]);
                if (tv > p[3] && tv < p[4]) b = std::fmax(b, q(tv));
            }
            return b;
        }
        case ICB_WAVE_EXPONENTIAL: {   // monotone in t between the start and end values
            const double v0 = std::fabs(p[0] + p[1]);
            const double v1 = std::fabs(p[0] + p[1] * std::exp(p[2] * (p[4] - p[3])));
            return std::fmax(v0, v1);
        }
        case ICB_WAVE_SINUSOIDAL: return std::fabs(p[0]) + std::fabs(p[1]);
        case ICB_WAVE_PWM:
        case ICB_WAVE_PULSED: return std::fmax(std::fabs(p[0]), std::fabs(p[1]));
        default: {
            double m = 0.0;
            for (int i = 0; i < w.n_points; ++i) m = std::fmax(m, std::fabs(w.values[i]));
            // Catmull-Rom: |h10|, |h11| <= 4/27 and |dt m| <= 2 max|v| keep the
            // spline within 1.6 max|v|
            return w.interp == ICB_INTERP_CUBIC ? 2.0 * m : m;
        }
    }
}

int check_waveform(const icb_waveform& w) {
    if (w.type < ICB_WAVE_CONSTANT || w.type > ICB_WAVE_ARBITRARY)
        return fail(ICB_ERR_INVALID_ARGUMENT, "unknown waveform type %d", w.type);
    for (int i = 0; i < 8; ++i)
        if (!std::isfinite(w.p[i])) return fail(ICB_ERR_INVALID_ARGUMENT, "waveform parameter %d is not finite", i);
    if (w.type == ICB_WAVE_ARBITRARY) {
        if (w.n_points < 1 || w.n_points > ICB_MAX_WAVE_POINTS)
            return fail(ICB_ERR_INVALID_ARGUMENT, "arbitrary waveform needs 1..%d points", ICB_MAX_WAVE_POINTS);
        if (w.interp < ICB_INTERP_LINEAR || w.interp > ICB_INTERP_CUBIC)
            return fail(ICB_ERR_INVALID_ARGUMENT, "unknown interpolation %d", w.interp);
        for (int i = 0; i < w.n_points; ++i) {
            if (!std::isfinite(w.times_s[i]) || !std::isfinite(w.values[i]))
                return fail(ICB_ERR_INVALID_ARGUMENT, "arbitrary waveform point %d is not finite", i);
            if (i > 0 && w.times_s[i] < w.times_s[i - 1])
                return fail(ICB_ERR_INVALID_ARGUMENT, "arbitrary waveform times must be ascending");
        }
    }
    if (!std::isfinite(wave_bound(w)))
        return fail(ICB_ERR_INVALID_ARGUMENT, "waveform is unbounded over its time range (give a finite end time)");
    return ICB_OK;
}

WaveConst wave_const(const icb_waveform& w) {
    WaveConst c;
    std::memset(&c, 0, sizeof(c));
    c.type = w.type;
    c.clamp = w.clamp;
    c.interp = w.interp;
    c.n = w.type == ICB_WAVE_ARBITRARY ? w.n_points : 0;
    for (int i = 0; i < 8; ++i) c.p[i] = w.p[i];
    for (int i = 0; i < c.n; ++i) { c.tt[i] = w.times_s[i]; c.vv[i] = w.values[i]; }
    return c;
}

// Field bound of an ensemble on the time-dependent table (triangle
// inequality over the axial, radial and AC terms; every waveform at its
// largest |value|).
double tf_bound(const EnsConst& C, const icb_ensemble_params& P, const TimeField& F, const double wb[ICB_N_CHANNELS]) {
    const double Rp = P.radius_m + kGeomEps;
    const double L = P.length_m;
    double ez = 0.0;
    double raxis = Rp;
    if (F.inst == ICB_INSTRUMENT_TIMS) {
        double m = std::fmax(std::fabs(F.tims_ei), std::fabs(F.tims_ef));
        for (int i = 0; i < F.tims_nodes; ++i) {
            m = std::fmax(m, std::fabs(F.tims_pi[i]));
            if (F.tims_final_profile) m = std::fmax(m, std::fabs(F.tims_pf[i]));
        }
        ez = m;
    } else if (F.inst == ICB_INSTRUMENT_LQIT) {
        ez = 2.0 * (wb[kChAxial] / (L * L)) * (0.5 * L + kGeomEps);
    } else {
        ez = wb[kChAxial] / L;
        raxis = std::sqrt(P.origin_m[0] * P.origin_m[0] + P.origin_m[1] * P.origin_m[1]) + Rp;
    }
    const double exy = 2.0 * (wb[kChQuad] + wb[kChRfV]) * raxis / (P.radius_m * P.radius_m);
    double e = ez + exy;
    if (F.inst == ICB_INSTRUMENT_LQIT) {
        double ac = 0.0;
        for (int a = 0; a < (F.ac_dipolar ? 2 : 1); ++a) {
            const double A = wb[kChAcA + 3 * a] * (F.ac_dipolar ? wb[kChAcR + 3 * a] : 1.0);
            if (A > kMinVoltage) ac += A / P.radius_m;
        }
        if (ac > 0.0) e = e + ac;
    }
    (void)C;
    return e;
}

// Per-ensemble constants exactly as the reference derives them.
// HSS mixture constants of one ensemble (a single gas becomes n = 1).
int build_mix(const icb_ensemble_params& P, MixConst& M) {
    std::memset(&M, 0, sizeof(M));
    const bool mixture = P.n_gas >= 2;
    if (P.n_gas > kMaxGas) return fail(ICB_ERR_INVALID_ARGUMENT, "at most %d gas components", kMaxGas);
    M.n = mixture ? P.n_gas : 1;
    for (int i = 0; i < M.n; ++i) {
        const double n = mixture ? P.gas_mix_density_m3[i] : P.gas_density_m3;
        const double m = mixture ? P.gas_mix_mass_kg[i] : P.gas_mass_kg;
        const double sg = mixture ? P.gas_mix_sigma_m2[i] : P.sigma_m2;
        if (!(n >= 0.0) || !(m > 0.0) || !(sg > 0.0))
            return fail(ICB_ERR_INVALID_ARGUMENT, "gas component %d needs density >= 0, mass > 0, sigma > 0", i);
        M.A[i] = n * sg * P.dt_s;
        M.sig_n[i] = std::sqrt(kBoltzmann * P.temperature_K / m);
        M.mean_th[i] = M.sig_n[i] * kMeanChi3;
        M.m[i] = m;
        M.fA[i] = static_cast<float>(M.A[i]);
        M.fsig_n[i] = static_cast<float>(M.sig_n[i]);
        M.fmean_th[i] = static_cast<float>(M.mean_th[i]);
        M.fm[i] = static_cast<float>(m);
    }
    return ICB_OK;
}

int build_ens_const(const icb_ensemble_params& P, EnsConst& C, int& field_kind, bool& mag, int coll) {
    std::memset(&C, 0, sizeof(C));
    if (!(P.length_m > 0.0) || !(P.radius_m > 0.0)) return fail(ICB_ERR_INVALID_ARGUMENT, "ensemble geometry needs length_m > 0 and radius_m > 0");
    if (!(P.dt_s > 0.0)) return fail(ICB_ERR_INVALID_ARGUMENT, "ensemble dt_s must be > 0");
    int kind = kFieldUniform;
    const bool rf = std::fabs(P.rf_voltage_V) > kMinVoltage;
    switch (P.instrument) {
        case ICB_INSTRUMENT_IMS:            // AnalyticalFieldModel.cpp:136-161
            C.E0[2] = P.axial_V / P.length_m;
            if (rf) kind = kFieldLinearRF;
            break;
        case ICB_INSTRUMENT_QUADRUPOLE_RF:  // AnalyticalFieldModel.cpp:219-248
            if (std::fabs(P.axial_V) > kMinVoltage) C.E0[2] = P.axial_V / P.length_m;
            if (rf) kind = kFieldLinearRF;
            break;
        case ICB_INSTRUMENT_FTICR: {        // AnalyticalFieldModel.cpp:174-186
            const double L = P.length_m, r = P.radius_m;
            const double d = std::sqrt((L * L / 8.0) + (r * r / 4.0));
            const double factor = P.radial_V / (d * d);
            C.G[0] = factor; C.G[1] = factor; C.G[2] = -2.0 * factor;
            C.c[2] = 0.5 * L;
            kind = kFieldLinear;
            break;
        }
        case ICB_INSTRUMENT_TIMS:           // TIMSAxialFieldModel.h (time-dependent field table)
            C.tf = 1;
            C.r0sq = P.radius_m * P.radius_m;
            kind = kFieldLinearRF;
            break;
        case ICB_INSTRUMENT_LQIT: {         // AnalyticalFieldModel.cpp:81-134 (unrotated cylinder)
            // RF quadrupole about the cylinder axis, axial well about L/2
            C.c[0] = P.origin_m[0];
            C.c[1] = P.origin_m[1];
            if (std::fabs(P.axial_V) > kMinVoltage) {
                const double L = P.length_m;
                const double alpha = P.axial_V / (L * L);
                C.G[2] = -2.0 * alpha;
                C.c[2] = P.origin_m[2] + 0.5 * L;
                kind = kFieldLinear;
            }
            // the single-axis drive is x alone, without a ramp
            for (int a = 0; a < (P.ac_dipolar ? 2 : 1); ++a) {
                const double A = P.ac_amplitude_V[a] * (P.ac_dipolar ? P.ac_ramp[a] : 1.0);
                if (!(P.ac_frequency_Hz[a] >= 0.0) || !std::isfinite(A))
                    return fail(ICB_ERR_INVALID_ARGUMENT, "LQIT AC drive %d needs a finite amplitude and frequency >= 0",
                                a);
                if (std::fabs(A) > kMinVoltage) {
                    C.ac = 1;
                    C.ac_amp[a] = -A / P.radius_m;
                    C.ac_omega[a] = 2.0 * M_PI * P.ac_frequency_Hz[a];
                    C.ac_phase[a] = P.ac_phase_rad[a];
                }
            }
            if (rf || C.ac) kind = kFieldLinearRF;
            break;
        }
        default:
            return fail(ICB_ERR_UNSUPPORTED, "instrument %d not supported", P.instrument);
    }
    if (rf) {
        C.rf = 1;
        C.rf_U0 = P.dc_quad_V;
        C.rf_V = P.rf_voltage_V;
        C.rf_omega = 2.0 * M_PI * P.rf_frequency_Hz;
        C.r0sq = P.radius_m * P.radius_m;
    }
    field_kind = std::max(field_kind, kind);
    if (P.magnetic_enabled) {
        C.magnetic = 1;
        for (int a = 0; a < 3; ++a) C.B[a] = P.B_T[a];
        if (P.B_T[0] != 0.0 || P.B_T[1] != 0.0 || P.B_T[2] != 0.0) mag = true;
    }
    C.ox = P.origin_m[0]; C.oy = P.origin_m[1]; C.oz = P.origin_m[2];
    C.zmax_local = P.length_m + kGeomEps;
    C.rmax2 = (P.radius_m + kGeomEps) * (P.radius_m + kGeomEps);
    C.rmax = P.radius_m + kGeomEps;
    C.dt = P.dt_s;
    if (coll != kCollNone) {
        if (!(P.gas_mass_kg > 0.0) || !(P.temperature_K > 0.0))
            return fail(ICB_ERR_INVALID_ARGUMENT, "collisions need gas_mass_kg > 0 and temperature_K > 0");
        if (!(P.gas_density_m3 >= 0.0)) return fail(ICB_ERR_INVALID_ARGUMENT, "collisions need gas_density_m3 >= 0");
        if (coll == kCollLangevin) {
            // nu = n pi |q| sqrt(alpha' / (4 pi eps0 mu)) (sigma_L v of DampingForce.cpp:170-176)
            if (!(P.gas_polarizability_m3 > 0.0))
                return fail(ICB_ERR_INVALID_ARGUMENT, "Langevin collisions need gas_polarizability_m3 > 0");
            C.A = 0.0;
            C.lang_c = P.gas_density_m3 * P.dt_s * M_PI * std::sqrt(P.gas_polarizability_m3 / (4.0 * M_PI * kEps0));
        } else if (coll == kCollIPMTable || coll == kCollIPMMLP || coll == kCollIPMQuad) {
            // event cross-section pi b_max^2 (InteractionPotentialCollisionHandler.cpp:443-447)
            if (!(P.ipm_bmax_m > 0.0))
                return fail(ICB_ERR_INVALID_ARGUMENT, "interaction-potential collisions need ipm_bmax_m > 0");
            C.A = P.gas_density_m3 * (M_PI * P.ipm_bmax_m * P.ipm_bmax_m) * P.dt_s;
        } else if (coll == kCollHSSMix && P.n_gas >= 2) {
            C.A = 0.0;   // the mixture's totals are set below
        } else {
            if (!(P.sigma_m2 > 0.0)) return fail(ICB_ERR_INVALID_ARGUMENT, "collisions need sigma_m2 > 0");
            C.A = P.gas_density_m3 * P.sigma_m2 * P.dt_s;
        }
        C.sig_n = std::sqrt(kBoltzmann * P.temperature_K / P.gas_mass_kg);
        C.mean_th = C.sig_n * kMeanChi3;
        C.m_gas = P.gas_mass_kg;
        // gas flow (EnvironmentConfig::gas_velocity_at): constant vectors here,
        // the parabolic profile per ion in the kernel
        if (P.flow_model != ICB_FLOW_CONSTANT && P.flow_model != ICB_FLOW_AXIAL_UNIFORM &&
            P.flow_model != ICB_FLOW_AXIAL_PARABOLIC)
            return fail(ICB_ERR_INVALID_ARGUMENT, "unknown flow_model %d", P.flow_model);
        if (P.flow_model == ICB_FLOW_AXIAL_UNIFORM && !(P.axial_flow_velocity_m_s >= 0.0))
            return fail(ICB_ERR_INVALID_ARGUMENT, "axial_flow_velocity_m_s must be >= 0 for axial_uniform flow");
        if (P.flow_model == ICB_FLOW_AXIAL_PARABOLIC && !(P.axial_flow_max_velocity_m_s >= 0.0))
            return fail(ICB_ERR_INVALID_ARGUMENT,
                        "axial_flow_max_velocity_m_s must be >= 0 for axial_parabolic flow");
        for (int a = 0; a < 3; ++a) C.ug[a] = P.gas_velocity_m_s[a];
        if (P.flow_model == ICB_FLOW_AXIAL_UNIFORM) {
            C.ug[0] = 0.0; C.ug[1] = 0.0; C.ug[2] = P.axial_flow_velocity_m_s;
        } else if (P.flow_model == ICB_FLOW_AXIAL_PARABOLIC) {
            C.ug[0] = 0.0; C.ug[1] = 0.0; C.ug[2] = 0.0;
            C.flow = 1;
            C.flow_umax = P.axial_flow_max_velocity_m_s;
            C.flow_r2 = P.radius_m * P.radius_m;
        }
        C.fA = static_cast<float>(C.A);
        C.fmean_th = static_cast<float>(C.mean_th);
        C.fsig_n = static_cast<float>(C.sig_n);
        C.fm_gas = static_cast<float>(C.m_gas);
        for (int a = 0; a < 3; ++a) C.fug[a] = static_cast<float>(C.ug[a]);
        if (coll == kCollHSSMix) {
            // clock totals of the mixture: A = sum A_i, A <|th|> = sum A_i <|th_i|>
            MixConst M;
            if (int r = build_mix(P, M)) return r;
            double A = 0.0, Am = 0.0;
            for (int i = 0; i < M.n; ++i) {
                A += M.A[i];
                Am += M.A[i] * M.mean_th[i];
            }
            C.A = A;
            C.mean_th = A > 0.0 ? Am / A : 0.0;
            C.fA = static_cast<float>(C.A);
            C.fmean_th = static_cast<float>(C.mean_th);
        }
    }
    C.zdet = P.detector_z_m;
    C.Emax = field_bound(C, P);
    return ICB_OK;
}

// Rebuild the time-dependent field table, the ensembles' tf flags and
// field bounds, and the handle's field kind from the waveforms and TIMS
// fields set so far; uploads the table when any ensemble uses it.
int rebuild_time_fields(icb_handle* h) {
    const size_t ne = h->ens.size();
    std::vector<TimeField> tfs(ne);
    bool any = false;
    for (size_t e = 0; e < ne; ++e) {
        const icb_ensemble_params& P = h->ens[e];
        EnsConst& C = h->ens_const[e];
        bool set = false;
        for (int c = 0; c < ICB_N_CHANNELS; ++c) set = set || h->wave_set[e * ICB_N_CHANNELS + c];
        const bool tims = P.instrument == ICB_INSTRUMENT_TIMS;
        C.tf = (set || tims) ? 1 : 0;
        double base;
        if (C.tf) {
            any = true;
            TimeField& F = tfs[e];
            std::memset(&F, 0, sizeof(F));
            F.inst = P.instrument;
            F.L = P.length_m;
            F.R = P.radius_m;
            F.r0sq = P.radius_m * P.radius_m;
            F.ox = P.origin_m[0]; F.oy = P.origin_m[1]; F.oz = P.origin_m[2];
            F.ac_dipolar = P.ac_dipolar ? 1 : 0;
            F.ac_phase[0] = P.ac_phase_rad[0];
            F.ac_phase[1] = P.ac_phase_rad[1];
            // channel constants (the TIMS ramp has none: built-in ramp)
            const double constants[ICB_N_CHANNELS] = {
                P.axial_V, P.dc_quad_V, P.rf_voltage_V, P.rf_frequency_Hz, 0.0,
                P.ac_amplitude_V[0], P.ac_frequency_Hz[0], P.ac_ramp[0],
                P.ac_amplitude_V[1], P.ac_frequency_Hz[1], P.ac_ramp[1]};
            double wb[ICB_N_CHANNELS];
            for (int c = 0; c < ICB_N_CHANNELS; ++c) {
                if (h->wave_set[e * ICB_N_CHANNELS + c]) {
                    const icb_waveform& w = h->waves[e * ICB_N_CHANNELS + c];
                    F.ch[c] = wave_const(w);
                    wb[c] = wave_bound(w);
                } else {
                    F.ch[c].type = kWaveConstant;
                    F.ch[c].p[0] = constants[c];
                    wb[c] = std::fabs(constants[c]);
                }
            }
            F.ramp_wave = h->wave_set[e * ICB_N_CHANNELS + ICB_CHANNEL_TIMS_RAMP_FRACTION];
            if (tims && h->tims_set[e]) {
                const icb_tims_field& T = h->tims[e];
                F.tims_mode = T.ramp_mode;
                F.tims_nodes = T.n_nodes;
                F.tims_final_profile = T.n_nodes > 0 && T.has_final_profile;
                F.tims_t0 = T.ramp_start_s;
                F.tims_t1 = T.ramp_end_s;
                F.tims_tau = T.ramp_tau_s;
                F.tims_ei = T.initial_uniform_V_m;
                F.tims_ef = T.final_uniform_V_m;
                for (int i = 0; i < T.n_nodes; ++i) {
                    F.tims_z[i] = T.z_positions_m[i];
                    F.tims_pi[i] = T.initial_profile_V_m[i];
                    F.tims_pf[i] = T.final_profile_V_m[i];
                    F.tims_zf[i] = static_cast<float>(T.z_positions_m[i]);
                    F.tims_pif[i] = static_cast<float>(T.initial_profile_V_m[i]);
                    F.tims_pff[i] = static_cast<float>(T.final_profile_V_m[i]);
                    const double dz = i + 1 < T.n_nodes ? T.z_positions_m[i + 1] - T.z_positions_m[i] : 0.0;
                    F.tims_idz[i] = dz > 0.0 ? static_cast<float>(1.0 / dz) : 0.0f;
                }
            }
            base = tf_bound(C, P, F, wb);
        } else {
            base = field_bound(C, P);
        }
        if (e == 0 && h->sc) {
            C.Emax = base + (C.Emax - h->sc_emax_base);
            h->sc_emax_base = base;
        } else {
            C.Emax = base;
        }
    }
    if (any != h->any_tf && !h->shape_tuned) {
        // launch shape of the time-dependent instance where neither the
        // caller nor icb_autotune chose one: the autotuner's optimum on the
        // TIMS workload (64-thread blocks, a 6-lane deferred batch, 8 steps
        // per vote: 1.05e11 ion-steps/s; 4 steps per vote gave 9.8e10)
        if (h->cfg.block_size <= 0) h->block = any ? 64 : 128;
        if (h->cfg.pending_threshold <= 0) h->pend = any ? 6u : 10u;
        if (h->cfg.steps_per_vote <= 0) h->spv = 8u;
    }
    h->any_tf = any;
    h->field_kind = any ? std::max(h->base_field_kind, static_cast<int>(kFieldLinearRF)) : h->base_field_kind;
    if (any) {
        ICB_CUDA(cudaStreamSynchronize(h->stream));
        if (h->tfield.n < ne) ICB_CUDA(h->tfield.alloc(ne));
        ICB_CUDA(cudaMemcpy(h->tfield.p, tfs.data(), ne * sizeof(TimeField), cudaMemcpyHostToDevice));
    }
    ++h->gen;
    return ICB_OK;
}

inline unsigned grid_for(uint64_t n, int block) { return static_cast<unsigned>((n + block - 1) / block); }

uint32_t tf_stride(const icb_handle* h) {
    return static_cast<uint32_t>(kTfRowScalars * (h->cfg.integrator == ICB_INTEGRATOR_RK4 ? 2 : 1));
}

// Room for the per-step field tables of launches of up to K steps (all
// ensembles, plus the time sequences); allocates outside stream capture only.
int ensure_tf_tab(icb_handle* h, uint32_t K, cudaStream_t st) {
    const size_t rows = static_cast<size_t>(K) + 1u;
    const size_t need = h->ens.size() * rows * (tf_stride(h) + 1u);
    if (h->tf_tab.n >= need) return ICB_OK;
    cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
    ICB_CUDA(cudaStreamIsCapturing(st, &cs));
    if (cs != cudaStreamCaptureStatusNone)
        return fail(ICB_ERR_STATE, "field table too small inside a stream capture");
    // the old table may still be read by this handle's queued work: wait
    // for the handle's own streams only (not the whole device)
    ICB_CUDA(cudaStreamSynchronize(st));
    ICB_CUDA(cudaStreamSynchronize(h->stream));
    if (h->copy_stream) ICB_CUDA(cudaStreamSynchronize(h->copy_stream));
    if (h->copy_back_stream) ICB_CUDA(cudaStreamSynchronize(h->copy_back_stream));
    for (cudaStream_t cs2 : h->chunk_streams) ICB_CUDA(cudaStreamSynchronize(cs2));
    ICB_CUDA(h->tf_tab.alloc(need));
    h->drop_graph();
    return ICB_OK;
}

// The time-only field scalars of every step of a K-step launch for the
// ensembles with a time-dependent field, built on `st` before the step
// kernels read them (stage 0 at t_k; RK4 adds the half step).
int enqueue_tf_tables(icb_handle* h, uint32_t K, cudaStream_t st) {
    if (!h->any_tf) return ICB_OK;
    if (int r = ensure_tf_tab(h, K, st)) return r;
    const uint32_t stride = tf_stride(h);
    const int n_ens = static_cast<int>(h->ens.size());
    double* tseq = h->tf_tab.p + h->ens.size() * (static_cast<size_t>(K) + 1u) * stride;
    for (int e0 = 0; e0 < n_ens; e0 += kMaxLaunchEns) {
        const int ne = std::min(kMaxLaunchEns, n_ens - e0);
        StepParams p;
        std::memset(&p, 0, sizeof(p));
        p.tfield = h->tfield.p;
        p.t_dev = h->t_dev.p;
        p.n_steps = K;
        p.ens_base = static_cast<uint32_t>(e0);
        p.n_ens = static_cast<uint32_t>(ne);
        for (int e = 0; e < ne; ++e) p.ens[e] = h->ens_const[static_cast<size_t>(e0 + e)];
        const cudaError_t te = launch_tf_table(p, h->tf_tab.p, tseq, stride, st);
        ++h->launches;
        if (te != cudaSuccess) return fail(ICB_ERR_CUDA, "field table launch: %s", cudaGetErrorString(te));
    }
    return ICB_OK;
}

// Step kernels for ions [lo, hi) (all ions by default); the field tables of
// a time-dependent field are built first unless the caller built them
// (build_tf = false).
int launch_step(icb_handle* h, uint32_t K, int do_push, int do_collide, int do_finalize, uint64_t lo = 0,
                uint64_t hi = ~0ull, cudaStream_t stream = nullptr, bool build_tf = true) {
    cudaStream_t st = stream ? stream : h->stream;
    if (build_tf) {
        if (int r = enqueue_tf_tables(h, K, st)) return r;
    }
    const int n_ens = static_cast<int>(h->ens.size());
    if ((h->coll == kCollIPMTable || h->coll == kCollIPMMLP || h->coll == kCollIPMQuad) && h->ipm_nE == 0)
        return fail(ICB_ERR_STATE, "interaction-potential collisions need icb_ipm_configure first");
    if (h->coll == kCollIPMMLP && !h->mlp_ready)
        return fail(ICB_ERR_STATE, "the learned deflection needs icb_ipm_set_mlp first");
    if (h->coll == kCollEHSS) {
        for (size_t e = 0; e < h->ens.size(); ++e)
            if (e >= h->ehss_host.size() || h->ehss_host[e].empty())
                return fail(ICB_ERR_STATE, "EHSS needs icb_ehss_set_geometry for ensemble %zu", e);
    }
    for (int e0 = 0; e0 < n_ens; e0 += kMaxLaunchEns) {
        const int ne = std::min(kMaxLaunchEns, n_ens - e0);
        auto clip = [&](uint64_t v) { return std::min(std::max(v, lo), hi); };
        const uint64_t b = clip(h->ens_off[static_cast<size_t>(e0)]);
        const uint64_t en = clip(h->ens_off[static_cast<size_t>(e0 + ne)]);
        if (en <= b) continue;
        StepParams p;
        std::memset(&p, 0, sizeof(p));
        p.x = h->x.p; p.y = h->y.p; p.z = h->z.p;
        p.xh = h->xh.p; p.xl = h->xl.p; p.yh = h->yh.p; p.yl = h->yl.p; p.zh = h->zh.p; p.zl = h->zl.p;
        p.vx = h->vx(); p.vy = h->vy(); p.vz = h->vz();
        p.clkS = h->fp64() ? static_cast<void*>(h->Sd.p) : static_cast<void*>(h->Sf.p);
        p.clkU = h->fp64() ? static_cast<void*>(h->Ud.p) : static_cast<void*>(h->Uf.p);
        p.clk_next = h->clk_next.p;
        p.clk_start = h->clk_start.p;
        p.mass = h->mass.p; p.charge = h->charge.p; p.flags = h->flags.p;
        p.t_death = h->t_death.p; p.t_arr = h->t_arr.p;
        p.birth = h->has_birth ? h->birth.p : nullptr;
        p.escx = h->sc ? sc_field(h->sc, 0) : nullptr;
        p.escy = h->sc ? sc_field(h->sc, 1) : nullptr;
        p.escz = h->sc ? sc_field(h->sc, 2) : nullptr;
        p.zprev = h->zprev.p;
        p.ipm_tab = h->ipm_tab.p;
        p.ipm_nE = h->ipm_nE;
        p.ipm_nb = h->ipm_nb;
        p.ipm_lnEmin = h->ipm_lnEmin;
        p.ipm_inv_dlnE = h->ipm_inv_dlnE;
        p.ipm_pot = h->ipm_pot;
        p.ipm_bmax = h->ipm_bmax;
        p.ipm_gl = h->ipm_gl;
        p.ipm_net_lnEmin = h->ipm_net_lnEmin;
        p.ipm_net_scale = h->ipm_net_scale;
        p.mlp_w2 = h->mlp_w2.p;
        p.mlp_f = h->mlp_f.p;
        p.mix = h->mix.p;
        p.tfield = h->tfield.p;
        p.ehss_atoms = h->ehss_atoms.p;
        p.ehss_off = h->ehss_off.p;
        p.ehss_rgas = h->ehss_rgas.p;
        p.counters = h->counters.p;
        p.step_dev = h->step_dev.p;
        p.t_dev = h->t_dev.p;
        p.first_id = h->first_id;
        p.seed = h->cfg.rng_seed;
        philox_round_keys(h->cfg.rng_seed, p.rk);
        p.n_steps = K;
        p.pend_threshold = h->pend;
        p.steps_per_vote = h->spv;
        p.jumps = (h->cfg.stepping == ICB_STEPPING_EVENTS && !h->fp64()) || h->cfg.stepping == ICB_STEPPING_EVENTS_ALL
                      ? 1u : 0u;
        p.subcycles = h->cfg.collision_subcycles > 1 ? static_cast<uint32_t>(h->cfg.collision_subcycles) : 1u;
        p.ens_base = static_cast<uint32_t>(e0);
        p.n_ens = static_cast<uint32_t>(ne);
        p.do_push = do_push; p.do_collide = do_collide; p.do_finalize = do_finalize;
        for (int e = 0; e <= ne; ++e) p.ens_off[e] = clip(h->ens_off[static_cast<size_t>(e0 + e)]);
        for (int e = 0; e < ne; ++e) {
            p.ens[e] = h->ens_const[static_cast<size_t>(e0 + e)];
            if (p.ens[e].flow) p.flows = 1u;
        }
        if (h->any_tf) {
            p.tf_tab = h->tf_tab.p;
            p.tf_stride = tf_stride(h);
        }
        if (h->cfg.collision_test == ICB_TEST_PER_STEP) {
            // the per-step kernel: fused steps only, none of the per-launch extras
            if (!(do_push && do_collide && do_finalize))
                return fail(ICB_ERR_UNSUPPORTED, "the per-step collision test runs fused steps only (icb_advance)");
            if (h->any_tf || h->sc)
                return fail(ICB_ERR_UNSUPPORTED, "the per-step collision test has no time-dependent field or space charge");
            // prepare_ions_for_integration finds nothing to remove after a
            // whole-population per-step launch (graphs replay their captured
            // parameters, so they always prepare)
            p.skip_prepare = (h->prep_ok && lo == 0 && hi >= h->n && !h->cfg.use_graphs) ? 1u : 0u;
            for (int e = 0; e < ne; ++e) {
                EnsConst& E = p.ens[e];
                E.sp_m = h->sp_m[static_cast<size_t>(e0 + e)];
                E.sp_q = h->sp_q[static_cast<size_t>(e0 + e)];
                if (E.sp_m > 0.0) {
                    // the device's load_consts arithmetic, once per launch
                    const double inv_m = 1.0 / E.sp_m;
                    for (int a = 0; a < 3; ++a) {
                        E.sp_a64[a] = (E.E0[a] * E.sp_q) / E.sp_m;
                        E.sp_a32[a] = (E.E0[a] * E.sp_q) * inv_m;
                        E.sp_fa[a] = static_cast<float>(E.sp_a32[a]);
                    }
                    E.sp_fh = static_cast<float>(E.dt * 0.5);
                    E.sp_fdt = static_cast<float>(E.dt);
                    E.sp_fAmean = static_cast<float>(E.A * E.mean_th);
                }
            }
            cudaError_t err1;
            switch (h->cfg.precision) {
                case ICB_PREC_FP64: err1 = launch_step1_fp64(h->coll, p, st); break;
                case ICB_PREC_MIXED: err1 = launch_step1_mixed(h->coll, p, st); break;
                default: err1 = launch_step1_hilo(h->coll, p, st); break;
            }
            ++h->launches;
            if (err1 != cudaSuccess) return fail(ICB_ERR_CUDA, "per-step kernel launch: %s", cudaGetErrorString(err1));
            continue;
        }
        const dim3 grid(grid_for(en - b, h->block)), block(static_cast<unsigned>(h->block));
        cudaError_t err;
        switch (h->cfg.precision) {
            case ICB_PREC_FP64: err = launch_step_fp64(h->cfg.integrator, h->coll, h->field_kind, h->magnetic, p, grid, block, st); break;
            case ICB_PREC_MIXED: err = launch_step_mixed(h->cfg.integrator, h->coll, h->field_kind, h->magnetic, p, grid, block, st); break;
            default: err = launch_step_hilo(h->cfg.integrator, h->coll, h->field_kind, h->magnetic, p, grid, block, st); break;
        }
        ++h->launches;
        if (err == cudaErrorNotSupported)
            return fail(ICB_ERR_UNSUPPORTED, "no kernel for precision %d integrator %d collision %d",
                        h->cfg.precision, h->cfg.integrator, h->cfg.collision_model);
        if (err != cudaSuccess) return fail(ICB_ERR_CUDA, "step kernel launch: %s", cudaGetErrorString(err));
    }
    if (h->cfg.collision_test == ICB_TEST_PER_STEP && lo == 0 && hi >= h->n) h->prep_ok = true;
    return ICB_OK;
}

// Space-charge field of the current positions (before a push).
int solve_space_charge(icb_handle* h) {
    std::string err;
    const int r = sc_solve(h->sc, h->x.p, h->y.p, h->z.p, h->charge.p, h->flags.p, h->n, h->stream, err);
    if (r != ICB_OK) return fail(r, "space charge: %s", err.c_str());
    h->launches += static_cast<uint64_t>(sc_kernel_count(h->sc));
    return ICB_OK;
}

// The launch sequence of icb_advance(n_steps): counter reset, then per chunk
// of at most K steps the fused step kernel(s) and the device clock update.
// The first n_timed chunks are bracketed by events for per-kernel timing.
int enqueue_advance(icb_handle* h, uint64_t n_steps, size_t n_timed) {
    cudaStream_t s = h->stream;
    ICB_CUDA(cudaMemsetAsync(h->counters.p, 0, kNumCounters * sizeof(unsigned long long), s));
    h->launches = 0;
    const int ne = static_cast<int>(h->ens.size());
    uint64_t left = n_steps;
    size_t j = 0;
    h->sc_timed = 0;
    while (left > 0) {
        // with space charge every launch advances one step, after the solve
        // of the field at the step's start positions
        const uint32_t K = h->sc ? 1u : static_cast<uint32_t>(std::min<uint64_t>(left, h->K));
        if (h->sc) {
            const bool timed = n_timed > 0 && h->sc_timed < 64;
            if (timed) ICB_CUDA(cudaEventRecord(h->sc_ev[2 * h->sc_timed], s));
            if (int r = solve_space_charge(h)) return r;
            if (timed) ICB_CUDA(cudaEventRecord(h->sc_ev[2 * h->sc_timed + 1], s));
            if (timed) ++h->sc_timed;
        }
        if (j < n_timed) ICB_CUDA(cudaEventRecord(h->kev[2 * j], s));
        if (int r = launch_step(h, K, 1, 1, 1)) return r;
        if (j < n_timed) ICB_CUDA(cudaEventRecord(h->kev[2 * j + 1], s));
        k_clock_advance<<<(ne + 127) / 128, 128, 0, s>>>(h->step_dev.p, h->t_dev.p, h->dt_dev.p, ne, K);
        ICB_CUDA(cudaGetLastError());
        ++h->launches;
        left -= K;
        ++j;
    }
    return ICB_OK;
}

int read_stats(icb_handle* h, icb_run_stats* st, uint64_t steps, size_t n_timed_launches) {
    unsigned long long c[kNumCounters];
    ICB_CUDA(cudaMemcpyAsync(c, h->counters.p, sizeof(c), cudaMemcpyDeviceToHost, h->stream));
    ICB_CUDA(cudaStreamSynchronize(h->stream));
    float ms = 0.f;
    ICB_CUDA(cudaEventElapsedTime(&ms, h->ev0, h->ev1));
    double kms = 0.0;
    for (size_t j = 0; j < n_timed_launches; ++j) {
        float m = 0.f;
        ICB_CUDA(cudaEventElapsedTime(&m, h->kev[2 * j], h->kev[2 * j + 1]));
        kms += m;
    }
    st->step_kernel_ms = kms;
    double scms = 0.0;
    for (size_t j = 0; j < h->sc_timed; ++j) {
        float m = 0.f;
        ICB_CUDA(cudaEventElapsedTime(&m, h->sc_ev[2 * j], h->sc_ev[2 * j + 1]));
        scms += m;
    }
    st->spacecharge_ms = scms;
    st->spacecharge_solves_timed = h->sc_timed;
    st->kernel_launches = h->launches;
    st->steps = steps;
    st->candidates = c[kCntCandidates];
    st->collisions = c[kCntCollisions];
    st->rate_overflows = c[kCntOverflow];
    st->deaths = c[kCntDeaths];
    st->arrivals = c[kCntArrivals];
    st->device_ms = static_cast<double>(ms);
    if (c[kCntStalls] != 0)
        return fail(ICB_ERR_CUDA, "per-step kernel: %llu staged tile copies did not complete within a second",
                    c[kCntStalls]);
    return ICB_OK;
}

template <class T>
void add_state(std::vector<std::pair<void*, size_t>>& v, DevBuf<T>& b) {
    if (b.p) v.emplace_back(static_cast<void*>(b.p), b.n * sizeof(T));
}

// Device buffers that a step changes (allocated ones only), for the
// autotuner's save/restore.
std::vector<std::pair<void*, size_t>> mutable_state(icb_handle* h) {
    std::vector<std::pair<void*, size_t>> v;
    add_state(v, h->x); add_state(v, h->y); add_state(v, h->z);
    add_state(v, h->xh); add_state(v, h->xl); add_state(v, h->yh);
    add_state(v, h->yl); add_state(v, h->zh); add_state(v, h->zl);
    add_state(v, h->vxd); add_state(v, h->vyd); add_state(v, h->vzd);
    add_state(v, h->vxf); add_state(v, h->vyf); add_state(v, h->vzf);
    add_state(v, h->Sd); add_state(v, h->Ud); add_state(v, h->Sf); add_state(v, h->Uf);
    add_state(v, h->clk_next); add_state(v, h->clk_start);
    add_state(v, h->flags); add_state(v, h->t_death); add_state(v, h->t_arr); add_state(v, h->zprev);
    add_state(v, h->step_dev); add_state(v, h->t_dev);
    return v;
}

}  // namespace

// ---------------------------------------------------------------------------
// C ABI
// ---------------------------------------------------------------------------
extern "C" {

int icb_abi_version(void) { return ICB_ABI_VERSION; }

const char* icb_last_error(void) { return g_last_error.c_str(); }

int icb_device_count(int* count) {
    if (!count) return fail(ICB_ERR_INVALID_ARGUMENT, "null count");
    int c = 0;
    cudaError_t e = cudaGetDeviceCount(&c);
    if (e != cudaSuccess) {
        *count = 0;
        return fail(ICB_ERR_NO_DEVICE, "cudaGetDeviceCount: %s", cudaGetErrorString(e));
    }
    *count = c;
    return ICB_OK;
}

int icb_create(const icb_config* cfg, icb_handle** out) {
    if (!cfg || !out) return fail(ICB_ERR_INVALID_ARGUMENT, "null config or output pointer");
    *out = nullptr;
    if (cfg->n_ensembles < 1 || cfg->n_ensembles > ICB_MAX_ENSEMBLES || !cfg->ensembles)
        return fail(ICB_ERR_INVALID_ARGUMENT, "n_ensembles must be in [1, %d] with a parameter array", ICB_MAX_ENSEMBLES);
    if (cfg->precision < ICB_PREC_FP64 || cfg->precision > ICB_PREC_MIXED_HILO)
        return fail(ICB_ERR_INVALID_ARGUMENT, "unknown precision %d", cfg->precision);
    if (cfg->integrator != ICB_INTEGRATOR_BORIS && cfg->integrator != ICB_INTEGRATOR_RK4)
        return fail(ICB_ERR_INVALID_ARGUMENT, "unknown integrator %d", cfg->integrator);
    if (cfg->precision == ICB_PREC_MIXED_HILO && cfg->integrator != ICB_INTEGRATOR_BORIS)
        return fail(ICB_ERR_UNSUPPORTED, "the hi/lo position variant is built for the Boris pusher only");
    int coll;
    switch (cfg->collision_model) {
        case ICB_COLLISION_NONE: coll = kCollNone; break;
        case ICB_COLLISION_HSS: {
            coll = kCollHSS;
            for (int32_t e = 0; e < cfg->n_ensembles; ++e)
                if (cfg->ensembles[e].n_gas >= 2) coll = kCollHSSMix;
            if (coll == kCollHSSMix && cfg->integrator != ICB_INTEGRATOR_BORIS)
                return fail(ICB_ERR_UNSUPPORTED, "HSS gas mixtures are built for the Boris pusher");
            break;
        }
        case ICB_COLLISION_EHSS:
            if (cfg->integrator != ICB_INTEGRATOR_BORIS)
                return fail(ICB_ERR_UNSUPPORTED, "EHSS collisions are built for the Boris pusher");
            coll = kCollEHSS;
            break;
        case ICB_COLLISION_HSS_PLAIN:
            if (cfg->integrator != ICB_INTEGRATOR_BORIS || cfg->precision != ICB_PREC_FP64)
                return fail(ICB_ERR_UNSUPPORTED, "the plain per-step HSS form is built for FP64 Boris");
            coll = kCollHSSPlain;
            break;
        case ICB_COLLISION_IPM_TABLE:
        case ICB_COLLISION_IPM_MLP:
        case ICB_COLLISION_IPM_QUAD:
            if (cfg->integrator != ICB_INTEGRATOR_BORIS)
                return fail(ICB_ERR_UNSUPPORTED, "interaction-potential collisions are built for the Boris pusher");
            coll = cfg->collision_model == ICB_COLLISION_IPM_TABLE ? kCollIPMTable
                 : cfg->collision_model == ICB_COLLISION_IPM_MLP   ? kCollIPMMLP
                                                                   : kCollIPMQuad;
            break;
        case ICB_COLLISION_LANGEVIN:
            if (cfg->integrator != ICB_INTEGRATOR_BORIS)
                return fail(ICB_ERR_UNSUPPORTED, "Langevin capture collisions are built for the Boris pusher");
            coll = kCollLangevin;
            break;
        default: return fail(ICB_ERR_UNSUPPORTED, "collision model %d not available", cfg->collision_model);
    }
    if (cfg->collision_subcycles < 0 || cfg->collision_subcycles > 1024)
        return fail(ICB_ERR_INVALID_ARGUMENT, "collision_subcycles must be in [0, 1024]");
    if (cfg->collision_subcycles > 1 && cfg->collision_model != ICB_COLLISION_HSS_PLAIN)
        return fail(ICB_ERR_UNSUPPORTED, "collision sub-steps need ICB_COLLISION_HSS_PLAIN");
    int ndev = 0;
    cudaError_t ce = cudaGetDeviceCount(&ndev);
    if (ce != cudaSuccess || ndev == 0) return fail(ICB_ERR_NO_DEVICE, "no CUDA device: %s", cudaGetErrorString(ce));
    if (cfg->device < 0 || cfg->device >= ndev) return fail(ICB_ERR_INVALID_ARGUMENT, "device %d out of range (%d devices)", cfg->device, ndev);
    std::unique_ptr<icb_handle> h(new icb_handle());
    h->cfg = *cfg;
    h->cfg.ensembles = nullptr;
    h->coll = coll;
    h->ens.assign(cfg->ensembles, cfg->ensembles + cfg->n_ensembles);
    h->ens_const.resize(h->ens.size());
    for (size_t e = 0; e < h->ens.size(); ++e) {
        int r = build_ens_const(h->ens[e], h->ens_const[e], h->field_kind, h->magnetic, coll);
        if (r != ICB_OK) return r;
    }
    std::vector<MixConst> mixes;
    if (coll == kCollHSSMix) {
        mixes.resize(h->ens.size());
        for (size_t e = 0; e < h->ens.size(); ++e)
            if (int r = build_mix(h->ens[e], mixes[e])) return r;
    }
    if (cfg->block_size > 0) {
        if (cfg->block_size % 32 != 0 || cfg->block_size > 128)
            return fail(ICB_ERR_INVALID_ARGUMENT, "block_size must be a multiple of 32 and <= 128");
        h->block = cfg->block_size;
    }
    if (cfg->steps_per_launch > 0) {
        if (cfg->steps_per_launch > static_cast<int32_t>(kMaxStepsPerLaunch))
            return fail(ICB_ERR_INVALID_ARGUMENT, "steps_per_launch must be <= %u", kMaxStepsPerLaunch);
        h->K = static_cast<uint32_t>(cfg->steps_per_launch);
    }
    // Deferred-collision batch per warp (lanes of 32): measured optimum with
    // 8 steps per vote.
    h->pend = 10u;
    if (cfg->pending_threshold > 0) h->pend = static_cast<uint32_t>(std::min(cfg->pending_threshold, 32));
    if (cfg->steps_per_vote > 0) h->spv = static_cast<uint32_t>(std::min(cfg->steps_per_vote, 64));
    if (cfg->stepping != ICB_STEPPING_EVENTS && cfg->stepping != ICB_STEPPING_PER_STEP &&
        cfg->stepping != ICB_STEPPING_EVENTS_ALL)
        return fail(ICB_ERR_INVALID_ARGUMENT, "stepping must be ICB_STEPPING_EVENTS, _PER_STEP or _EVENTS_ALL");
    if (cfg->collision_test != ICB_TEST_CLOCK && cfg->collision_test != ICB_TEST_PER_STEP)
        return fail(ICB_ERR_INVALID_ARGUMENT, "collision_test must be ICB_TEST_CLOCK or ICB_TEST_PER_STEP");
    if (cfg->collision_test == ICB_TEST_PER_STEP) {
        // the per-step kernel's physics (icb_step1.cuh)
        if (cfg->integrator != ICB_INTEGRATOR_BORIS || (coll != kCollNone && coll != kCollHSS))
            return fail(ICB_ERR_UNSUPPORTED, "the per-step collision test runs Boris with hard-sphere or no collisions");
        if (h->field_kind != kFieldUniform || h->magnetic)
            return fail(ICB_ERR_UNSUPPORTED, "the per-step collision test runs uniform electric fields without B");
        for (const auto& c : h->ens_const)
            if (c.flow) return fail(ICB_ERR_UNSUPPORTED, "the per-step collision test needs a constant or axial-uniform gas flow");
        if (cfg->steps_per_launch <= 0) h->K = 1u;   // the state goes back to HBM after every step
    }
    ICB_CUDA(cudaSetDevice(cfg->device));
    ICB_CUDA(cudaStreamCreateWithFlags(&h->own_stream, cudaStreamNonBlocking));
    h->stream = h->own_stream;
    ICB_CUDA(cudaEventCreate(&h->ev0));
    ICB_CUDA(cudaEventCreate(&h->ev1));
    ICB_CUDA(h->counters.alloc(kNumCounters));
    ICB_CUDA(h->step_dev.alloc(1));
    ICB_CUDA(h->t_dev.alloc(h->ens.size()));
    ICB_CUDA(h->dt_dev.alloc(h->ens.size()));
    std::vector<double> dts(h->ens.size()), zeros(h->ens.size(), 0.0);
    for (size_t e = 0; e < h->ens.size(); ++e) dts[e] = h->ens[e].dt_s;
    ICB_CUDA(cudaMemcpy(h->dt_dev.p, dts.data(), dts.size() * sizeof(double), cudaMemcpyHostToDevice));
    ICB_CUDA(cudaMemcpy(h->t_dev.p, zeros.data(), zeros.size() * sizeof(double), cudaMemcpyHostToDevice));
    ICB_CUDA(cudaMemset(h->step_dev.p, 0, sizeof(unsigned long long)));
    ICB_CUDA(cudaMemset(h->counters.p, 0, kNumCounters * sizeof(unsigned long long)));
    ICB_CUDA(h->mom_out.alloc(h->ens.size() * ICB_N_MOMENTS));
    if (!mixes.empty()) {
        ICB_CUDA(h->mix.alloc(mixes.size()));
        ICB_CUDA(cudaMemcpy(h->mix.p, mixes.data(), mixes.size() * sizeof(MixConst), cudaMemcpyHostToDevice));
    }
    h->base_field_kind = h->field_kind;
    h->waves.assign(h->ens.size() * ICB_N_CHANNELS, icb_waveform{});
    h->wave_set.assign(h->ens.size() * ICB_N_CHANNELS, 0);
    h->tims.assign(h->ens.size(), icb_tims_field{});
    h->tims_set.assign(h->ens.size(), 0);
    if (int r = rebuild_time_fields(h.get())) return r;
    *out = h.release();
    return ICB_OK;
}

int icb_destroy(icb_handle* h) {
    if (!h) return ICB_OK;
    cudaSetDevice(h->cfg.device);
    if (h->stream) cudaStreamSynchronize(h->stream);
    delete h;
    return ICB_OK;
}

int icb_set_stream(icb_handle* h, void* cuda_stream) {
    if (int r = check_handle(h)) return r;
    h->stream = cuda_stream ? static_cast<cudaStream_t>(cuda_stream) : h->own_stream;
    ++h->gen;
    return ICB_OK;
}

int icb_synchronize(icb_handle* h) {
    if (int r = check_handle(h)) return r;
    ICB_CUDA(cudaStreamSynchronize(h->stream));
    return ICB_OK;
}

uint64_t icb_ion_count(icb_handle* h) { return h ? h->n : 0; }

int icb_upload_ions(icb_handle* h, uint64_t n,
                    const double* x, const double* y, const double* z,
                    const double* vx, const double* vy, const double* vz,
                    const double* mass_kg, const double* charge_C,
                    const uint8_t* active, const double* birth_time_s,
                    const uint64_t* ens_offsets, uint64_t first_ion_id) {
    if (int r = check_handle(h)) return r;
    h->prep_ok = false;
    if (n == 0) return fail(ICB_ERR_INVALID_ARGUMENT, "no ions");
    if (!x || !y || !z || !vx || !vy || !vz || !mass_kg || !charge_C || !active)
        return fail(ICB_ERR_INVALID_ARGUMENT, "state arrays must not be NULL");
    if (first_ion_id + n > (1ull << 32)) return fail(ICB_ERR_INVALID_ARGUMENT, "ion ids must fit in 32 bits");
    const size_t ne = h->ens.size();
    std::vector<uint64_t> off(ne + 1);
    if (ens_offsets) {
        for (size_t e = 0; e <= ne; ++e) off[e] = ens_offsets[e];
        if (off[0] != 0 || off[ne] != n) return fail(ICB_ERR_INVALID_ARGUMENT, "ens_offsets must start at 0 and end at n");
        for (size_t e = 0; e < ne; ++e)
            if (off[e + 1] < off[e]) return fail(ICB_ERR_INVALID_ARGUMENT, "ens_offsets must be non-decreasing");
    } else {
        if (ne != 1) return fail(ICB_ERR_INVALID_ARGUMENT, "ens_offsets required with %zu ensembles", ne);
        off[0] = 0; off[1] = n;
    }
    for (uint64_t i = 0; i < n; ++i) {
        if (!(mass_kg[i] > 0.0)) return fail(ICB_ERR_INVALID_ARGUMENT, "ion %llu: mass must be > 0", static_cast<unsigned long long>(i));
    }
    if (h->cfg.collision_test == ICB_TEST_PER_STEP && birth_time_s)
        return fail(ICB_ERR_UNSUPPORTED, "the per-step collision test has no births (birth_time_s must be NULL)");
    // the species of each ensemble when all its ions share mass and charge
    // (the per-step kernel then reads neither per-ion array)
    h->sp_m.assign(ne, 0.0);
    h->sp_q.assign(ne, 0.0);
    for (size_t e = 0; e < ne; ++e) {
        if (off[e + 1] == off[e]) continue;
        const double m0 = mass_kg[off[e]], q0 = charge_C[off[e]];
        bool same = true;
        for (uint64_t i = off[e]; same && i < off[e + 1]; ++i) same = mass_kg[i] == m0 && charge_C[i] == q0;
        if (same) { h->sp_m[e] = m0; h->sp_q[e] = q0; }
    }
    ICB_CUDA(cudaStreamSynchronize(h->stream));
    if (h->n != n) {
        const bool f64 = h->fp64(), hl = h->hilo();
        ICB_CUDA(h->x.alloc(hl ? 0 : n)); ICB_CUDA(h->y.alloc(hl ? 0 : n)); ICB_CUDA(h->z.alloc(hl ? 0 : n));
        ICB_CUDA(h->xh.alloc(hl ? n : 0)); ICB_CUDA(h->xl.alloc(hl ? n : 0));
        ICB_CUDA(h->yh.alloc(hl ? n : 0)); ICB_CUDA(h->yl.alloc(hl ? n : 0));
        ICB_CUDA(h->zh.alloc(hl ? n : 0)); ICB_CUDA(h->zl.alloc(hl ? n : 0));
        ICB_CUDA(h->vxd.alloc(f64 ? n : 0)); ICB_CUDA(h->vyd.alloc(f64 ? n : 0)); ICB_CUDA(h->vzd.alloc(f64 ? n : 0));
        ICB_CUDA(h->vxf.alloc(f64 ? 0 : n)); ICB_CUDA(h->vyf.alloc(f64 ? 0 : n)); ICB_CUDA(h->vzf.alloc(f64 ? 0 : n));
        const bool clk = h->coll != kCollNone;
        ICB_CUDA(h->Sd.alloc(clk && f64 ? n : 0)); ICB_CUDA(h->Ud.alloc(clk && f64 ? n : 0));
        ICB_CUDA(h->Sf.alloc(clk && !f64 ? n : 0)); ICB_CUDA(h->Uf.alloc(clk && !f64 ? n : 0));
        // event-step arrays of the skip clock (read by the Boris kernels only)
        ICB_CUDA(h->clk_next.alloc(clk ? n : 0)); ICB_CUDA(h->clk_start.alloc(clk ? n : 0));
        ICB_CUDA(h->xr.alloc(n)); ICB_CUDA(h->yr.alloc(n)); ICB_CUDA(h->zr.alloc(n));
        ICB_CUDA(h->mass.alloc(n)); ICB_CUDA(h->charge.alloc(n));
        ICB_CUDA(h->t_death.alloc(n)); ICB_CUDA(h->t_arr.alloc(n)); ICB_CUDA(h->birth.alloc(n));
        ICB_CUDA(h->zprev.alloc(n));
        ICB_CUDA(h->flags.alloc(n)); ICB_CUDA(h->active_stage.alloc(n));
        ICB_CUDA(h->stage.alloc(f64 ? 0 : n));
        h->n = n;
    }
    h->first_id = first_ion_id;
    ++h->gen;
    h->ens_off = off;
    cudaStream_t s = h->stream;
    const unsigned g = grid_for(n, 256);
    const size_t bytes = n * sizeof(double);
    // positions
    const double* pos[3] = {x, y, z};
    DevBuf<double>* pd[3] = {&h->x, &h->y, &h->z};
    DevBuf<float>* ph[3] = {&h->xh, &h->yh, &h->zh};
    DevBuf<float>* pl[3] = {&h->xl, &h->yl, &h->zl};
    for (int a = 0; a < 3; ++a) {
        if (h->hilo()) {
            ICB_CUDA(cudaMemcpyAsync(h->stage.p, pos[a], bytes, cudaMemcpyHostToDevice, s));
            k_to_hilo<<<g, 256, 0, s>>>(h->stage.p, ph[a]->p, pl[a]->p, n);
            ICB_CUDA(cudaGetLastError());
        } else {
            ICB_CUDA(cudaMemcpyAsync(pd[a]->p, pos[a], bytes, cudaMemcpyHostToDevice, s));
        }
    }
    DevBuf<double>* pr[3] = {&h->xr, &h->yr, &h->zr};
    for (int a = 0; a < 3; ++a) ICB_CUDA(cudaMemcpyAsync(pr[a]->p, pos[a], bytes, cudaMemcpyHostToDevice, s));
    const double* vel[3] = {vx, vy, vz};
    DevBuf<double>* vd[3] = {&h->vxd, &h->vyd, &h->vzd};
    DevBuf<float>* vf[3] = {&h->vxf, &h->vyf, &h->vzf};
    for (int a = 0; a < 3; ++a) {
        if (h->fp64()) {
            ICB_CUDA(cudaMemcpyAsync(vd[a]->p, vel[a], bytes, cudaMemcpyHostToDevice, s));
        } else {
            ICB_CUDA(cudaMemcpyAsync(h->stage.p, vel[a], bytes, cudaMemcpyHostToDevice, s));
            k_to_float<<<g, 256, 0, s>>>(h->stage.p, vf[a]->p, n);
            ICB_CUDA(cudaGetLastError());
        }
    }
    ICB_CUDA(cudaMemcpyAsync(h->mass.p, mass_kg, bytes, cudaMemcpyHostToDevice, s));
    ICB_CUDA(cudaMemcpyAsync(h->charge.p, charge_C, bytes, cudaMemcpyHostToDevice, s));
    ICB_CUDA(cudaMemcpyAsync(h->active_stage.p, active, n, cudaMemcpyHostToDevice, s));
    h->has_birth = birth_time_s != nullptr;
    if (birth_time_s) ICB_CUDA(cudaMemcpyAsync(h->birth.p, birth_time_s, bytes, cudaMemcpyHostToDevice, s));
    k_flags_in<<<g, 256, 0, s>>>(h->active_stage.p, h->has_birth ? h->birth.p : nullptr, h->flags.p, h->t_death.p, h->t_arr.p, n);
    ICB_CUDA(cudaGetLastError());
    if (h->coll != kCollNone) {
        const int skip = h->skip_clock() ? 1 : 0;
        if (h->fp64())
            k_clock_init<double><<<g, 256, 0, s>>>(h->Sd.p, h->Ud.p, h->clk_next.p, h->clk_start.p, n, first_ion_id,
                                                   h->cfg.rng_seed, skip);
        else
            k_clock_init<float><<<g, 256, 0, s>>>(h->Sf.p, h->Uf.p, h->clk_next.p, h->clk_start.p, n, first_ion_id,
                                                  h->cfg.rng_seed, skip);
        ICB_CUDA(cudaGetLastError());
    }
    // moment work items: slices of <= kMomItemIons ions, never crossing an ensemble
    std::vector<MomItem> items;
    std::vector<int> item_off(ne + 1, 0);
    for (size_t e = 0; e < ne; ++e) {
        item_off[e] = static_cast<int>(items.size());
        for (uint64_t b = off[e]; b < off[e + 1]; b += kMomItemIons)
            items.push_back(MomItem{b, std::min<uint64_t>(off[e + 1], b + kMomItemIons)});
    }
    item_off[ne] = static_cast<int>(items.size());
    h->n_mom_items = static_cast<int>(items.size());
    ICB_CUDA(h->mom_items.alloc(std::max<size_t>(items.size(), 1)));
    ICB_CUDA(h->mom_item_off.alloc(ne + 1));
    ICB_CUDA(h->mom_partials.alloc(std::max<size_t>(items.size(), 1) * ICB_N_MOMENTS));
    if (!items.empty()) ICB_CUDA(cudaMemcpyAsync(h->mom_items.p, items.data(), items.size() * sizeof(MomItem), cudaMemcpyHostToDevice, s));
    ICB_CUDA(cudaMemcpyAsync(h->mom_item_off.p, item_off.data(), item_off.size() * sizeof(int), cudaMemcpyHostToDevice, s));
    ICB_CUDA(cudaStreamSynchronize(s));
    return ICB_OK;
}

int icb_update_state(icb_handle* h, const double* x, const double* y, const double* z,
                     const double* vx, const double* vy, const double* vz, const uint8_t* active) {
    if (int r = check_handle(h)) return r;
    h->prep_ok = false;
    if (h->n == 0) return fail(ICB_ERR_STATE, "no ions uploaded");
    cudaStream_t s = h->stream;
    const uint64_t n = h->n;
    const unsigned g = grid_for(n, 256);
    const size_t bytes = n * sizeof(double);
    const double* pos[3] = {x, y, z};
    DevBuf<double>* pd[3] = {&h->x, &h->y, &h->z};
    DevBuf<float>* ph[3] = {&h->xh, &h->yh, &h->zh};
    DevBuf<float>* pl[3] = {&h->xl, &h->yl, &h->zl};
    for (int a = 0; a < 3; ++a) {
        if (!pos[a]) continue;
        if (h->hilo()) {
            ICB_CUDA(cudaMemcpyAsync(h->stage.p, pos[a], bytes, cudaMemcpyHostToDevice, s));
            k_to_hilo<<<g, 256, 0, s>>>(h->stage.p, ph[a]->p, pl[a]->p, n);
            ICB_CUDA(cudaGetLastError());
        } else {
            ICB_CUDA(cudaMemcpyAsync(pd[a]->p, pos[a], bytes, cudaMemcpyHostToDevice, s));
        }
    }
    const double* vel[3] = {vx, vy, vz};
    DevBuf<double>* vd[3] = {&h->vxd, &h->vyd, &h->vzd};
    DevBuf<float>* vf[3] = {&h->vxf, &h->vyf, &h->vzf};
    for (int a = 0; a < 3; ++a) {
        if (!vel[a]) continue;
        if (h->fp64()) {
            ICB_CUDA(cudaMemcpyAsync(vd[a]->p, vel[a], bytes, cudaMemcpyHostToDevice, s));
        } else {
            ICB_CUDA(cudaMemcpyAsync(h->stage.p, vel[a], bytes, cudaMemcpyHostToDevice, s));
            k_to_float<<<g, 256, 0, s>>>(h->stage.p, vf[a]->p, n);
            ICB_CUDA(cudaGetLastError());
        }
    }
    if (active) {
        ICB_CUDA(cudaMemcpyAsync(h->active_stage.p, active, n, cudaMemcpyHostToDevice, s));
        k_flags_update<<<g, 256, 0, s>>>(h->active_stage.p, h->flags.p, n);
        ICB_CUDA(cudaGetLastError());
    }
    return ICB_OK;
}

int icb_download_ions(icb_handle* h, double* x, double* y, double* z,
                      double* vx, double* vy, double* vz,
                      uint8_t* active, double* death_time_s, double* arrival_time_s) {
    if (int r = check_handle(h)) return r;
    if (h->n == 0) return fail(ICB_ERR_STATE, "no ions uploaded");
    cudaStream_t s = h->stream;
    const uint64_t n = h->n;
    const unsigned g = grid_for(n, 256);
    const size_t bytes = n * sizeof(double);
    double* pos[3] = {x, y, z};
    DevBuf<double>* pd[3] = {&h->x, &h->y, &h->z};
    DevBuf<float>* ph[3] = {&h->xh, &h->yh, &h->zh};
    DevBuf<float>* pl[3] = {&h->xl, &h->yl, &h->zl};
    for (int a = 0; a < 3; ++a) {
        if (!pos[a]) continue;
        if (h->hilo()) {
            k_from_hilo<<<g, 256, 0, s>>>(ph[a]->p, pl[a]->p, h->stage.p, n);
            ICB_CUDA(cudaGetLastError());
            ICB_CUDA(cudaMemcpyAsync(pos[a], h->stage.p, bytes, cudaMemcpyDeviceToHost, s));
            ICB_CUDA(cudaStreamSynchronize(s));
        } else {
            ICB_CUDA(cudaMemcpyAsync(pos[a], pd[a]->p, bytes, cudaMemcpyDeviceToHost, s));
        }
    }
    double* vel[3] = {vx, vy, vz};
    DevBuf<double>* vd[3] = {&h->vxd, &h->vyd, &h->vzd};
    DevBuf<float>* vf[3] = {&h->vxf, &h->vyf, &h->vzf};
    for (int a = 0; a < 3; ++a) {
        if (!vel[a]) continue;
        if (h->fp64()) {
            ICB_CUDA(cudaMemcpyAsync(vel[a], vd[a]->p, bytes, cudaMemcpyDeviceToHost, s));
        } else {
            k_from_float<<<g, 256, 0, s>>>(vf[a]->p, h->stage.p, n);
            ICB_CUDA(cudaGetLastError());
            ICB_CUDA(cudaMemcpyAsync(vel[a], h->stage.p, bytes, cudaMemcpyDeviceToHost, s));
            ICB_CUDA(cudaStreamSynchronize(s));
        }
    }
    if (active) {
        k_flags_out<<<g, 256, 0, s>>>(h->flags.p, h->active_stage.p, n);
        ICB_CUDA(cudaGetLastError());
        ICB_CUDA(cudaMemcpyAsync(active, h->active_stage.p, n, cudaMemcpyDeviceToHost, s));
    }
    if (death_time_s) ICB_CUDA(cudaMemcpyAsync(death_time_s, h->t_death.p, bytes, cudaMemcpyDeviceToHost, s));
    if (arrival_time_s) ICB_CUDA(cudaMemcpyAsync(arrival_time_s, h->t_arr.p, bytes, cudaMemcpyDeviceToHost, s));
    ICB_CUDA(cudaStreamSynchronize(s));
    return ICB_OK;
}

int icb_advance(icb_handle* h, uint64_t n_steps, icb_run_stats* stats) {
    if (int r = check_handle(h)) return r;
    if (h->n == 0) return fail(ICB_ERR_STATE, "no ions uploaded");
    // Philox counters and clock events use 31-bit global step indices.
    if (h->host_step + n_steps >= (1ull << 31))
        return fail(ICB_ERR_INVALID_ARGUMENT, "runs are limited to 2^31 engine steps");
    h->host_step += n_steps;
    cudaStream_t s = h->stream;
    if (h->cfg.use_graphs) {
        // Replay one captured graph per distinct n_steps: counters reset, the
        // fused step launches and the device clock updates.
        if (!h->graph || h->graph_steps != n_steps || h->graph_gen != h->gen) {
            h->drop_graph();
            // Captured on the handle's own non-blocking stream (capture is
            // not allowed on the legacy default stream); replayed on h->stream.
            cudaGraph_t g = nullptr;
            if (h->any_tf) {
                if (int r = ensure_tf_tab(h, static_cast<uint32_t>(std::min<uint64_t>(n_steps, h->K)), s)) return r;
            }
            ICB_CUDA(cudaStreamBeginCapture(h->own_stream, cudaStreamCaptureModeThreadLocal));
            h->stream = h->own_stream;
            int r = enqueue_advance(h, n_steps, 0);
            h->stream = s;
            cudaError_t ce = cudaStreamEndCapture(h->own_stream, &g);
            if (r != ICB_OK) { if (g) cudaGraphDestroy(g); return r; }
            if (ce != cudaSuccess) return fail(ICB_ERR_CUDA, "graph capture: %s", cudaGetErrorString(ce));
            ce = cudaGraphInstantiate(&h->graph, g, 0);
            cudaGraphDestroy(g);
            if (ce != cudaSuccess) { h->graph = nullptr; return fail(ICB_ERR_CUDA, "cudaGraphInstantiate: %s", cudaGetErrorString(ce)); }
            h->graph_steps = n_steps;
            h->graph_gen = h->gen;
            h->graph_launches = h->launches;
        }
        ICB_CUDA(cudaEventRecord(h->ev0, s));
        ICB_CUDA(cudaGraphLaunch(h->graph, s));
        ICB_CUDA(cudaEventRecord(h->ev1, s));
        h->launches = h->graph_launches;
        if (stats) {
            if (int r = read_stats(h, stats, n_steps, 0)) return r;
            stats->step_kernel_ms = stats->device_ms;   // kernels are not timed one by one inside a graph
        }
        return ICB_OK;
    }
    ICB_CUDA(cudaEventRecord(h->ev0, s));
    // Per-launch events around the step kernels when statistics are asked
    // for (at most 64 launches are timed individually per call).
    const uint64_t k_eff = h->sc ? 1u : h->K;
    const size_t n_launch = static_cast<size_t>((n_steps + k_eff - 1) / k_eff);
    const size_t n_timed = stats ? std::min<size_t>(n_launch, 64) : 0;
    while (h->kev.size() < 2 * n_timed || (h->sc && h->sc_ev.size() < 128)) {
        cudaEvent_t e;
        ICB_CUDA(cudaEventCreate(&e));
        if (h->kev.size() < 2 * n_timed) h->kev.push_back(e);
        else h->sc_ev.push_back(e);
    }
    if (int r = enqueue_advance(h, n_steps, n_timed)) return r;
    ICB_CUDA(cudaEventRecord(h->ev1, s));
    if (stats) return read_stats(h, stats, n_steps, n_timed);
    return ICB_OK;
}

// Field bound of the collision majorant: 4 x the largest space-charge field
// of the current state (own ions, and the peers' ions when set).
int sc_auto_bound(icb_handle* h) {
    std::string err;
    const int r = sc_solve(h->sc, h->x.p, h->y.p, h->z.p, h->charge.p, h->flags.p, h->n, h->stream, err);
    if (r != ICB_OK) return fail(r, "space charge: %s", err.c_str());
    std::vector<double> e[3];
    for (int a = 0; a < 3; ++a) {
        e[a].resize(h->n);
        ICB_CUDA(cudaMemcpyAsync(e[a].data(), sc_field(h->sc, a), h->n * sizeof(double), cudaMemcpyDeviceToHost,
                                 h->stream));
    }
    ICB_CUDA(cudaStreamSynchronize(h->stream));
    double mx = 0.0;
    for (uint64_t i = 0; i < h->n; ++i)
        mx = std::max(mx, std::sqrt(e[0][i] * e[0][i] + e[1][i] * e[1][i] + e[2][i] * e[2][i]));
    h->ens_const[0].Emax = h->sc_emax_base + 4.0 * mx;
    ++h->gen;
    return ICB_OK;
}

int icb_spacecharge_configure(icb_handle* h, const icb_spacecharge_config* cfg) {
    if (int r = check_handle(h)) return r;
    if (!cfg) return fail(ICB_ERR_INVALID_ARGUMENT, "null space-charge config");
    ICB_CUDA(cudaStreamSynchronize(h->stream));
    if (h->sc) {
        sc_destroy(h->sc);
        h->sc = nullptr;
        h->ens_const[0].Emax = h->sc_emax_base;
    }
    ++h->gen;
    if (cfg->mode == ICB_SC_OFF) return ICB_OK;
    if (h->n == 0) return fail(ICB_ERR_STATE, "upload the ions before configuring space charge");
    if (h->ens.size() != 1) return fail(ICB_ERR_UNSUPPORTED, "space charge couples one ensemble's ions: use one ensemble");
    if (h->cfg.integrator != ICB_INTEGRATOR_BORIS)
        return fail(ICB_ERR_UNSUPPORTED, "space charge needs the Boris pusher (RK4 refreshes it per stage)");
    if (h->hilo()) return fail(ICB_ERR_UNSUPPORTED, "space charge is built for the FP64 and mixed position forms");
    std::string err;
    SpaceChargeSolver* sc = nullptr;
    // the float forms (and an FP64 handle that asks for it) run the mesh and
    // the particle-particle sums in single precision
    int r = sc_create(*cfg, h->n, !h->fp64() || cfg->solver_fp32 != 0, h->stream, &sc, err);
    if (r != ICB_OK) return fail(r, "space charge: %s", err.c_str());
    h->sc = sc;
    h->sc_emax_base = h->ens_const[0].Emax;
    h->sc_bound_auto = !(cfg->field_bound_V_m > 0.0);
    h->sc_peers_bounded = false;
    h->sc_peer_ptr = nullptr;
    h->sc_peer_n = h->sc_peer_skip_b = h->sc_peer_skip_n = 0;
    if (!h->sc_bound_auto) {
        h->ens_const[0].Emax = h->sc_emax_base + cfg->field_bound_V_m;
        return ICB_OK;
    }
    return sc_auto_bound(h);
}

// Space charge across devices: other devices' ions join this handle's solve.
int icb_spacecharge_set_peers(icb_handle* h, uint64_t n, const double* xyzq_device, uint64_t skip_begin,
                              uint64_t skip_count) {
    if (int r = check_handle(h)) return r;
    if (!h->sc) return fail(ICB_ERR_STATE, "space charge is not configured");
    std::string err;
    const int r = sc_set_peers(h->sc, xyzq_device, n, skip_begin, skip_count, h->stream, err);
    if (r != ICB_OK) return fail(r, "space charge: %s", err.c_str());
    const void* ptr = n ? static_cast<const void*>(xyzq_device) : nullptr;
    if (ptr != h->sc_peer_ptr || n != h->sc_peer_n || skip_begin != h->sc_peer_skip_b ||
        skip_count != h->sc_peer_skip_n) {
        // a captured graph holds the solver's launch parameters
        ++h->gen;
        h->sc_peer_ptr = ptr;
        h->sc_peer_n = n;
        h->sc_peer_skip_b = skip_begin;
        h->sc_peer_skip_n = skip_count;
    }
    // the automatic field bound is taken again with the peers' ions, once
    if (n > 0 && h->sc_bound_auto && !h->sc_peers_bounded) {
        h->sc_peers_bounded = true;
        return sc_auto_bound(h);
    }
    return ICB_OK;
}

int icb_spacecharge_export(icb_handle* h, double* xyzq_device) {
    if (int r = check_handle(h)) return r;
    if (h->n == 0) return fail(ICB_ERR_STATE, "no ions uploaded");
    if (h->hilo()) return fail(ICB_ERR_UNSUPPORTED, "space charge is built for the FP64 and mixed position forms");
    std::string err;
    const int r = sc_export(h->x.p, h->y.p, h->z.p, h->charge.p, h->flags.p, h->n, xyzq_device, h->stream, err);
    if (r != ICB_OK) return fail(r, "space charge: %s", err.c_str());
    return ICB_OK;
}

int icb_ipm_configure(icb_handle* h, const icb_ipm_config* cfg) {
    if (int r = check_handle(h)) return r;
    if (!cfg) return fail(ICB_ERR_INVALID_ARGUMENT, "null IPM config");
    if (cfg->n_E < 2 || cfg->n_b < 2 || cfg->n_E > 16384 || cfg->n_b > 16384)
        return fail(ICB_ERR_INVALID_ARGUMENT, "IPM table needs 2 <= n_E, n_b <= 16384");
    if (!(cfg->E_min_J > 0.0) || !(cfg->E_max_J > cfg->E_min_J) || !(cfg->b_max_m > 0.0))
        return fail(ICB_ERR_INVALID_ARGUMENT, "IPM table needs 0 < E_min < E_max and b_max > 0");
    const bool net_default = cfg->net_E_min_J == 0.0 && cfg->net_E_max_J == 0.0;
    const double net_lo = net_default ? cfg->E_min_J : cfg->net_E_min_J;
    const double net_hi = net_default ? cfg->E_max_J : cfg->net_E_max_J;
    if (!(net_lo > 0.0) || !(net_hi > net_lo))
        return fail(ICB_ERR_INVALID_ARGUMENT, "IPM network range needs 0 < net_E_min < net_E_max");
    for (const auto& e : h->ens)
        if (std::fabs(e.ipm_bmax_m - cfg->b_max_m) > 1e-12 * cfg->b_max_m)
            return fail(ICB_ERR_INVALID_ARGUMENT, "b_max_m must equal every ensemble's ipm_bmax_m");
    std::string err;
    IpmPotential P{};
    if (int r = ipm_potential_from(cfg->potential, P, err)) return fail(r, "%s", err.c_str());
    ICB_CUDA(cudaStreamSynchronize(h->stream));
    ICB_CUDA(h->ipm_tab.alloc(static_cast<size_t>(cfg->n_E) * cfg->n_b));
    int r = ipm_build_table(h->cfg.device, P, cfg->n_E, cfg->n_b, cfg->E_min_J, cfg->E_max_J, cfg->b_max_m,
                            h->ipm_tab.p, h->stream, err);
    if (r != ICB_OK) {
        h->ipm_nE = 0;
        return fail(r, "%s", err.c_str());
    }
    h->ipm_nE = cfg->n_E;
    h->ipm_nb = cfg->n_b;
    h->ipm_lnEmin = std::log(cfg->E_min_J);
    h->ipm_inv_dlnE = (cfg->n_E - 1) / (std::log(cfg->E_max_J) - h->ipm_lnEmin);
    h->ipm_bmax = cfg->b_max_m;
    h->ipm_Emin = cfg->E_min_J;
    h->ipm_Emax = cfg->E_max_J;
    if (int r2 = ipm_gl_nodes(h->cfg.device, &h->ipm_gl, err)) return fail(r2, "%s", err.c_str());
    h->ipm_pot = P;
    h->ipm_net_lnEmin = std::log(net_lo);
    h->ipm_net_scale = 2.0 / (std::log(net_hi) - h->ipm_net_lnEmin);
    ++h->gen;
    return ICB_OK;
}

int icb_ehss_set_geometry(icb_handle* h, int32_t ensemble, int32_t n_atoms, const double* centers_m,
                          const double* radii_m, double gas_radius_m) {
    if (int r = check_handle(h)) return r;
    if (ensemble < 0 || static_cast<size_t>(ensemble) >= h->ens.size())
        return fail(ICB_ERR_INVALID_ARGUMENT, "ensemble %d out of range", ensemble);
    if (n_atoms < 1 || n_atoms > 100000 || !centers_m || !radii_m)
        return fail(ICB_ERR_INVALID_ARGUMENT, "EHSS geometry needs 1..100000 atoms with centres and radii");
    if (!(gas_radius_m >= 0.0)) return fail(ICB_ERR_INVALID_ARGUMENT, "gas_radius_m must be >= 0");
    for (int32_t j = 0; j < n_atoms; ++j)
        if (!(radii_m[j] > 0.0)) return fail(ICB_ERR_INVALID_ARGUMENT, "atom %d: radius must be > 0", j);
    h->ehss_host.resize(h->ens.size());
    h->ehss_rgas_host.resize(h->ens.size(), 0.0);
    auto& atoms = h->ehss_host[static_cast<size_t>(ensemble)];
    atoms.resize(static_cast<size_t>(n_atoms));
    for (int32_t j = 0; j < n_atoms; ++j)
        atoms[static_cast<size_t>(j)] = make_double4(centers_m[3 * j], centers_m[3 * j + 1], centers_m[3 * j + 2],
                                                     radii_m[j]);
    h->ehss_rgas_host[static_cast<size_t>(ensemble)] = gas_radius_m;
    std::vector<double4> all;
    std::vector<int32_t> off(1, 0);
    for (const auto& v : h->ehss_host) {
        all.insert(all.end(), v.begin(), v.end());
        off.push_back(static_cast<int32_t>(all.size()));
    }
    ICB_CUDA(cudaStreamSynchronize(h->stream));
    ICB_CUDA(h->ehss_atoms.alloc(all.size()));
    ICB_CUDA(h->ehss_off.alloc(off.size()));
    ICB_CUDA(h->ehss_rgas.alloc(h->ehss_rgas_host.size()));
    ICB_CUDA(cudaMemcpy(h->ehss_atoms.p, all.data(), all.size() * sizeof(double4), cudaMemcpyHostToDevice));
    ICB_CUDA(cudaMemcpy(h->ehss_off.p, off.data(), off.size() * sizeof(int32_t), cudaMemcpyHostToDevice));
    ICB_CUDA(cudaMemcpy(h->ehss_rgas.p, h->ehss_rgas_host.data(), h->ehss_rgas_host.size() * sizeof(double),
                        cudaMemcpyHostToDevice));
    ++h->gen;
    return ICB_OK;
}

int icb_set_waveform(icb_handle* h, int32_t ensemble, int32_t channel, const icb_waveform* w) {
    if (int r = check_handle(h)) return r;
    if (ensemble < 0 || static_cast<size_t>(ensemble) >= h->ens.size())
        return fail(ICB_ERR_INVALID_ARGUMENT, "ensemble %d out of range", ensemble);
    if (channel < 0 || channel >= ICB_N_CHANNELS) return fail(ICB_ERR_INVALID_ARGUMENT, "unknown channel %d", channel);
    const int inst = h->ens[static_cast<size_t>(ensemble)].instrument;
    if (inst == ICB_INSTRUMENT_FTICR)
        return fail(ICB_ERR_UNSUPPORTED, "the FTICR field evaluates its voltages once (t = 0): no waveforms");
    if (channel == ICB_CHANNEL_TIMS_RAMP_FRACTION && inst != ICB_INSTRUMENT_TIMS)
        return fail(ICB_ERR_INVALID_ARGUMENT, "the TIMS ramp channel needs instrument TIMS");
    if (channel >= ICB_CHANNEL_AC_X_AMPLITUDE_V) {
        if (inst != ICB_INSTRUMENT_LQIT) return fail(ICB_ERR_INVALID_ARGUMENT, "the AC channels need an LQIT");
        const bool dip = h->ens[static_cast<size_t>(ensemble)].ac_dipolar != 0;
        if (!dip && (channel == ICB_CHANNEL_AC_X_RAMP || channel >= ICB_CHANNEL_AC_Y_AMPLITUDE_V))
            return fail(ICB_ERR_INVALID_ARGUMENT, "ramp and y-axis AC channels need the two-axis dipolar drive");
    }
    if (w) {
        if (int r = check_waveform(*w)) return r;
    }
    const size_t slot = static_cast<size_t>(ensemble) * ICB_N_CHANNELS + static_cast<size_t>(channel);
    if (w) h->waves[slot] = *w;
    h->wave_set[slot] = w ? 1 : 0;
    return rebuild_time_fields(h);
}

int icb_set_tims_field(icb_handle* h, int32_t ensemble, const icb_tims_field* f) {
    if (int r = check_handle(h)) return r;
    if (ensemble < 0 || static_cast<size_t>(ensemble) >= h->ens.size())
        return fail(ICB_ERR_INVALID_ARGUMENT, "ensemble %d out of range", ensemble);
    if (h->ens[static_cast<size_t>(ensemble)].instrument != ICB_INSTRUMENT_TIMS)
        return fail(ICB_ERR_INVALID_ARGUMENT, "ensemble %d is not a TIMS domain", ensemble);
    if (f) {
        // TIMSFieldConfig::validate (FieldsConfig.h:262-300)
        if (f->ramp_mode != ICB_TIMS_RAMP_LINEAR && f->ramp_mode != ICB_TIMS_RAMP_EXPONENTIAL)
            return fail(ICB_ERR_INVALID_ARGUMENT, "TIMS ramp_mode must be linear or exponential");
        const double sc[5] = {f->initial_uniform_V_m, f->final_uniform_V_m, f->ramp_start_s, f->ramp_end_s,
                              f->ramp_tau_s};
        for (double v : sc)
            if (!std::isfinite(v)) return fail(ICB_ERR_INVALID_ARGUMENT, "TIMS parameters must be finite");
        if (f->ramp_end_s < f->ramp_start_s) return fail(ICB_ERR_INVALID_ARGUMENT, "TIMS ramp_end_s must be >= ramp_start_s");
        if (f->ramp_mode == ICB_TIMS_RAMP_EXPONENTIAL && !(f->ramp_tau_s > 0.0))
            return fail(ICB_ERR_INVALID_ARGUMENT, "TIMS ramp_tau_s must be > 0 for exponential mode");
        if (f->n_nodes != 0 && (f->n_nodes < 2 || f->n_nodes > ICB_MAX_WAVE_POINTS))
            return fail(ICB_ERR_INVALID_ARGUMENT, "TIMS profiles need 2..%d nodes", ICB_MAX_WAVE_POINTS);
        for (int i = 0; i < f->n_nodes; ++i) {
            if (!std::isfinite(f->z_positions_m[i]) || !std::isfinite(f->initial_profile_V_m[i]) ||
                (f->has_final_profile && !std::isfinite(f->final_profile_V_m[i])))
                return fail(ICB_ERR_INVALID_ARGUMENT, "TIMS profile node %d is not finite", i);
            if (i > 0 && f->z_positions_m[i] < f->z_positions_m[i - 1])
                return fail(ICB_ERR_INVALID_ARGUMENT, "TIMS z_positions_m must be ascending");
        }
        h->tims[static_cast<size_t>(ensemble)] = *f;
    }
    h->tims_set[static_cast<size_t>(ensemble)] = f ? 1 : 0;
    return rebuild_time_fields(h);
}

int icb_ipm_set_mlp(icb_handle* h, const float* params) {
    if (int r = check_handle(h)) return r;
    if (!params) return fail(ICB_ERR_INVALID_ARGUMENT, "null params");
    std::vector<uint32_t> frag;
    std::vector<float> fb;
    mlp_pack(params, frag, fb);
    ICB_CUDA(cudaStreamSynchronize(h->stream));
    ICB_CUDA(h->mlp_w2.alloc(frag.size()));
    ICB_CUDA(h->mlp_f.alloc(fb.size()));
    ICB_CUDA(cudaMemcpy(h->mlp_w2.p, frag.data(), frag.size() * sizeof(uint32_t), cudaMemcpyHostToDevice));
    ICB_CUDA(cudaMemcpy(h->mlp_f.p, fb.data(), fb.size() * sizeof(float), cudaMemcpyHostToDevice));
    h->mlp_ready = true;
    ++h->gen;
    return ICB_OK;
}

int icb_ipm_table(icb_handle* h, float* out) {
    if (int r = check_handle(h)) return r;
    if (h->ipm_nE == 0) return fail(ICB_ERR_STATE, "no IPM table");
    if (!out) return fail(ICB_ERR_INVALID_ARGUMENT, "null output");
    ICB_CUDA(cudaMemcpyAsync(out, h->ipm_tab.p, h->ipm_tab.n * sizeof(float), cudaMemcpyDeviceToHost, h->stream));
    ICB_CUDA(cudaStreamSynchronize(h->stream));
    return ICB_OK;
}

int icb_spacecharge_field(icb_handle* h, double* ex, double* ey, double* ez) {
    if (int r = check_handle(h)) return r;
    if (!h->sc) return fail(ICB_ERR_STATE, "space charge is not configured");
    h->launches = 0;
    if (int r = solve_space_charge(h)) return r;
    double* out[3] = {ex, ey, ez};
    for (int a = 0; a < 3; ++a)
        if (out[a])
            ICB_CUDA(cudaMemcpyAsync(out[a], sc_field(h->sc, a), h->n * sizeof(double), cudaMemcpyDeviceToHost,
                                     h->stream));
    ICB_CUDA(cudaStreamSynchronize(h->stream));
    return ICB_OK;
}

int icb_autotune(icb_handle* h, uint64_t trial_steps, icb_tuning* out) {
    if (int r = check_handle(h)) return r;
    if (h->n == 0) return fail(ICB_ERR_STATE, "no ions uploaded");
    if (h->cfg.collision_test == ICB_TEST_PER_STEP)
        return fail(ICB_ERR_UNSUPPORTED, "the per-step kernel has a fixed launch shape");
    if (trial_steps == 0) trial_steps = 500;
    if (trial_steps > 100000) return fail(ICB_ERR_INVALID_ARGUMENT, "trial_steps must be <= 100000");
    if (h->host_step + trial_steps >= (1ull << 31))
        return fail(ICB_ERR_INVALID_ARGUMENT, "runs are limited to 2^31 engine steps");
    cudaStream_t s = h->stream;
    // Save the state once; every trial starts from it and it is put back at
    // the end, so the handle's trajectory is unchanged by tuning.
    const auto bufs = mutable_state(h);
    size_t total = 0;
    for (const auto& b : bufs) total += (b.second + 255) & ~size_t(255);
    DevBuf<uint8_t> saved;
    ICB_CUDA(saved.alloc(total));
    auto copy_all = [&](bool save) -> cudaError_t {
        size_t off = 0;
        for (const auto& b : bufs) {
            void* dst = save ? static_cast<void*>(saved.p + off) : b.first;
            const void* src = save ? b.first : static_cast<const void*>(saved.p + off);
            cudaError_t e = cudaMemcpyAsync(dst, src, b.second, cudaMemcpyDeviceToDevice, s);
            if (e != cudaSuccess) return e;
            off += (b.second + 255) & ~size_t(255);
        }
        return cudaSuccess;
    };
    ICB_CUDA(copy_all(true));
    const int blk0 = h->block;
    const uint32_t spv0 = h->spv, pend0 = h->pend;
    const int blocks[] = {64, 128};
    const uint32_t spvs[] = {4, 8, 16};
    const uint32_t pends[] = {6, 10, 14};
    const bool coll = h->coll != kCollNone;
    double best_ms = 1e300;
    int best_blk = blk0;
    uint32_t best_spv = spv0, best_pend = pend0;
    int trials = 0;
    auto timed = [&](int blk, uint32_t spv, uint32_t pend, float* ms) -> int {
        h->block = blk; h->spv = spv; h->pend = pend;
        ICB_CUDA(copy_all(false));
        ICB_CUDA(cudaEventRecord(h->ev0, s));
        if (int r = enqueue_advance(h, trial_steps, 0)) return r;
        ICB_CUDA(cudaEventRecord(h->ev1, s));
        ICB_CUDA(cudaEventSynchronize(h->ev1));
        ICB_CUDA(cudaEventElapsedTime(ms, h->ev0, h->ev1));
        return ICB_OK;
    };
    int rc = ICB_OK;
    float ms = 0.f;
    rc = timed(blk0, spv0, pend0, &ms);   // warm-up
    for (int blk : blocks) {
        for (uint32_t spv : spvs) {
            for (uint32_t pend : pends) {
                if (rc != ICB_OK) break;
                if (!coll && pend != pends[0]) continue;   // the threshold only matters with collisions
                const uint32_t pe = coll ? pend : pend0;
                float m0 = 0.f, m1 = 0.f;
                if ((rc = timed(blk, spv, pe, &m0)) != ICB_OK) break;
                if ((rc = timed(blk, spv, pe, &m1)) != ICB_OK) break;
                ++trials;
                const double m = std::min(m0, m1);
                if (m < best_ms) { best_ms = m; best_blk = blk; best_spv = spv; best_pend = pe; }
            }
        }
    }
    // Back to the saved state with the chosen shape (or the old one on error).
    if (rc == ICB_OK) { h->block = best_blk; h->spv = best_spv; h->pend = best_pend; h->shape_tuned = true; }
    else { h->block = blk0; h->spv = spv0; h->pend = pend0; }
    ICB_CUDA(copy_all(false));
    ICB_CUDA(cudaStreamSynchronize(s));
    ++h->gen;
    if (rc != ICB_OK) return rc;
    if (out) {
        std::memset(out, 0, sizeof(*out));
        out->block_size = h->block;
        out->steps_per_vote = static_cast<int32_t>(h->spv);
        out->pending_threshold = static_cast<int32_t>(h->pend);
        out->steps_per_launch = static_cast<int32_t>(h->K);
        out->trials = trials;
        out->ion_steps_per_s = static_cast<double>(h->n) * static_cast<double>(trial_steps) / (best_ms * 1e-3);
    }
    return ICB_OK;
}

int icb_advance_host(icb_handle* h, uint64_t n_steps, int n_chunks, double* x, double* y, double* z, double* vx,
                     double* vy, double* vz, uint8_t* active, icb_run_stats* stats) {
    if (int r = check_handle(h)) return r;
    h->prep_ok = false;
    if (h->n == 0) return fail(ICB_ERR_STATE, "no ions uploaded");
    if (!x || !y || !z || !vx || !vy || !vz || !active) return fail(ICB_ERR_INVALID_ARGUMENT, "null state array");
    if (n_chunks < 1 || n_chunks > 64) return fail(ICB_ERR_INVALID_ARGUMENT, "n_chunks must be in [1, 64]");
    if (n_steps == 0) return fail(ICB_ERR_INVALID_ARGUMENT, "n_steps must be > 0");
    // the overlapped form needs one launch per chunk and independent ions
    // (its chunks launch directly, also on a handle that replays
    // icb_advance through CUDA graphs)
    if (n_chunks == 1 || n_steps > h->K || h->sc || h->hilo()) {
        if (int r = icb_update_state(h, x, y, z, vx, vy, vz, active)) return r;
        if (int r = icb_advance(h, n_steps, stats)) return r;
        return icb_download_ions(h, x, y, z, vx, vy, vz, active, nullptr, nullptr);
    }
    if (h->host_step + n_steps >= (1ull << 31))
        return fail(ICB_ERR_INVALID_ARGUMENT, "runs are limited to 2^31 engine steps");
    const uint64_t n = h->n;
    const bool f64 = h->fp64();
    if (!h->copy_stream) ICB_CUDA(cudaStreamCreateWithFlags(&h->copy_stream, cudaStreamNonBlocking));
    if (!h->copy_back_stream) ICB_CUDA(cudaStreamCreateWithFlags(&h->copy_back_stream, cudaStreamNonBlocking));
    while (h->chunk_streams.size() < static_cast<size_t>(n_chunks)) {
        cudaStream_t cst;
        ICB_CUDA(cudaStreamCreateWithFlags(&cst, cudaStreamNonBlocking));
        h->chunk_streams.push_back(cst);
    }
    while (h->hev.size() < static_cast<size_t>(2 * n_chunks + 1)) {
        cudaEvent_t e;
        ICB_CUDA(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
        h->hev.push_back(e);
    }
    if (!f64 && h->hstage.n < 3 * n) ICB_CUDA(h->hstage.alloc(3 * n));
    cudaStream_t s = h->stream, cs = h->copy_stream, bs = h->copy_back_stream;
    double* pos[3] = {x, y, z};
    double* vel[3] = {vx, vy, vz};
    double* pd[3] = {h->x.p, h->y.p, h->z.p};
    double* vd[3] = {h->vxd.p, h->vyd.p, h->vzd.p};
    float* vf[3] = {h->vxf.p, h->vyf.p, h->vzf.p};
    // chunk c = ions [lim[c], lim[c+1]), boundaries on 256-ion multiples
    std::vector<uint64_t> lim(static_cast<size_t>(n_chunks) + 1);
    for (int c = 0; c <= n_chunks; ++c)
        lim[static_cast<size_t>(c)] = c == n_chunks ? n : std::min<uint64_t>(n, ((n * c / n_chunks) + 255) & ~255ull);
    h->host_step += n_steps;
    h->launches = 0;
    h->sc_timed = 0;
    ICB_CUDA(cudaMemsetAsync(h->counters.p, 0, kNumCounters * sizeof(unsigned long long), s));
    ICB_CUDA(cudaEventRecord(h->ev0, s));
    ICB_CUDA(cudaEventRecord(h->hev[2 * n_chunks], s));
    ICB_CUDA(cudaStreamWaitEvent(cs, h->hev[2 * n_chunks], 0));   // earlier work on the state is done
    // Chunk by chunk: inputs on the copy stream, steps on the chunk's own
    // stream (so a chunk's blocks fill the SMs while the previous chunk's
    // last blocks finish), results on the copy-back stream.  Queued in chunk
    // order, the first chunk's steps start as soon as its inputs are in.
    // one field table for all chunks, ahead of every chunk's steps
    if (int r = enqueue_tf_tables(h, static_cast<uint32_t>(n_steps), cs)) return r;
    for (int c = 0; c < n_chunks; ++c) {
        const uint64_t a = lim[static_cast<size_t>(c)], b = lim[static_cast<size_t>(c) + 1], cnt = b - a;
        if (cnt == 0) continue;
        for (int k = 0; k < 3; ++k) {
            ICB_CUDA(cudaMemcpyAsync(pd[k] + a, pos[k] + a, cnt * sizeof(double), cudaMemcpyHostToDevice, cs));
            double* dst = f64 ? vd[k] + a : h->hstage.p + k * n + a;
            ICB_CUDA(cudaMemcpyAsync(dst, vel[k] + a, cnt * sizeof(double), cudaMemcpyHostToDevice, cs));
        }
        ICB_CUDA(cudaMemcpyAsync(h->active_stage.p + a, active + a, cnt, cudaMemcpyHostToDevice, cs));
        ICB_CUDA(cudaEventRecord(h->hev[2 * c], cs));
        const unsigned g = grid_for(cnt, 256);
        cudaStream_t ks = h->chunk_streams[static_cast<size_t>(c)];
        ICB_CUDA(cudaStreamWaitEvent(ks, h->hev[2 * c], 0));
        double* stage = f64 ? nullptr : h->hstage.p + a;
        k_chunk_in<<<g, 256, 0, ks>>>(stage, n, f64 ? nullptr : vf[0] + a, f64 ? nullptr : vf[1] + a,
                                      f64 ? nullptr : vf[2] + a, h->active_stage.p + a, h->flags.p + a, cnt);
        ICB_CUDA(cudaGetLastError());
        if (int r = launch_step(h, static_cast<uint32_t>(n_steps), 1, 1, 1, a, b, ks, false)) return r;
        k_chunk_out<<<g, 256, 0, ks>>>(f64 ? nullptr : vf[0] + a, f64 ? nullptr : vf[1] + a, f64 ? nullptr : vf[2] + a,
                                       stage, n, h->flags.p + a, h->active_stage.p + a, cnt);
        ICB_CUDA(cudaGetLastError());
        h->launches += 2;
        ICB_CUDA(cudaEventRecord(h->hev[2 * c + 1], ks));
        ICB_CUDA(cudaStreamWaitEvent(bs, h->hev[2 * c + 1], 0));
        for (int k = 0; k < 3; ++k) {
            ICB_CUDA(cudaMemcpyAsync(pos[k] + a, pd[k] + a, cnt * sizeof(double), cudaMemcpyDeviceToHost, bs));
            const double* src = f64 ? vd[k] + a : h->hstage.p + k * n + a;
            ICB_CUDA(cudaMemcpyAsync(vel[k] + a, src, cnt * sizeof(double), cudaMemcpyDeviceToHost, bs));
        }
        ICB_CUDA(cudaMemcpyAsync(active + a, h->active_stage.p + a, cnt, cudaMemcpyDeviceToHost, bs));
    }
    // the copy-back stream has waited for every chunk's steps: the clock
    // advance follows them (and the copies) through it
    ICB_CUDA(cudaEventRecord(h->hev[2 * n_chunks], bs));
    ICB_CUDA(cudaStreamWaitEvent(s, h->hev[2 * n_chunks], 0));
    const int ne = static_cast<int>(h->ens.size());
    k_clock_advance<<<(ne + 127) / 128, 128, 0, s>>>(h->step_dev.p, h->t_dev.p, h->dt_dev.p, ne,
                                                      static_cast<uint32_t>(n_steps));
    ICB_CUDA(cudaGetLastError());
    ++h->launches;
    ICB_CUDA(cudaEventRecord(h->ev1, s));
    if (stats) return read_stats(h, stats, n_steps, 0);
    ICB_CUDA(cudaStreamSynchronize(s));
    return ICB_OK;
}

static int single_part(icb_handle* h, int push, int collide, int finalize, icb_run_stats* stats) {
    if (int r = check_handle(h)) return r;
    if (h->n == 0) return fail(ICB_ERR_STATE, "no ions uploaded");
    if (h->host_step + 1 >= (1ull << 31))
        return fail(ICB_ERR_INVALID_ARGUMENT, "runs are limited to 2^31 engine steps");
    if (finalize) h->host_step += 1;
    cudaStream_t s = h->stream;
    ICB_CUDA(cudaMemsetAsync(h->counters.p, 0, kNumCounters * sizeof(unsigned long long), s));
    ICB_CUDA(cudaEventRecord(h->ev0, s));
    h->launches = 0;
    h->sc_timed = 0;
    if (push && h->sc) {
        if (int r = solve_space_charge(h)) return r;
    }
    if (int r = launch_step(h, 1, push, collide, finalize)) return r;
    if (finalize) {
        const int ne = static_cast<int>(h->ens.size());
        k_clock_advance<<<(ne + 127) / 128, 128, 0, s>>>(h->step_dev.p, h->t_dev.p, h->dt_dev.p, ne, 1);
        ICB_CUDA(cudaGetLastError());
        ++h->launches;
    }
    ICB_CUDA(cudaEventRecord(h->ev1, s));
    if (stats) return read_stats(h, stats, finalize ? 1 : 0, 0);
    return ICB_OK;
}

int icb_push(icb_handle* h) { return single_part(h, 1, 0, 0, nullptr); }
int icb_collide(icb_handle* h, icb_run_stats* stats) { return single_part(h, 0, 1, 0, stats); }
int icb_finalize(icb_handle* h, icb_run_stats* stats) { return single_part(h, 0, 0, 1, stats); }

int icb_get_clock(icb_handle* h, uint64_t* step, double* time_s) {
    if (int r = check_handle(h)) return r;
    unsigned long long st = 0;
    ICB_CUDA(cudaMemcpyAsync(&st, h->step_dev.p, sizeof(st), cudaMemcpyDeviceToHost, h->stream));
    if (time_s) ICB_CUDA(cudaMemcpyAsync(time_s, h->t_dev.p, h->ens.size() * sizeof(double), cudaMemcpyDeviceToHost, h->stream));
    ICB_CUDA(cudaStreamSynchronize(h->stream));
    if (step) *step = st;
    return ICB_OK;
}

int icb_set_clock(icb_handle* h, uint64_t step, const double* time_s) {
    if (int r = check_handle(h)) return r;
    if (step >= (1ull << 31)) return fail(ICB_ERR_INVALID_ARGUMENT, "step index must be < 2^31");
    h->host_step = step;
    unsigned long long st = step;
    ICB_CUDA(cudaMemcpyAsync(h->step_dev.p, &st, sizeof(st), cudaMemcpyHostToDevice, h->stream));
    if (time_s) ICB_CUDA(cudaMemcpyAsync(h->t_dev.p, time_s, h->ens.size() * sizeof(double), cudaMemcpyHostToDevice, h->stream));
    ICB_CUDA(cudaStreamSynchronize(h->stream));
    return ICB_OK;
}

int icb_moments(icb_handle* h, double* out) {
    if (int r = check_handle(h)) return r;
    if (!out) return fail(ICB_ERR_INVALID_ARGUMENT, "null output");
    if (h->n == 0) return fail(ICB_ERR_STATE, "no ions uploaded");
    cudaStream_t s = h->stream;
    const int ne = static_cast<int>(h->ens.size());
    if (h->n_mom_items > 0) {
        if (h->fp64()) {
            k_moments_partial<double, false><<<h->n_mom_items, 256, 0, s>>>(
                h->mom_items.p, h->x.p, h->y.p, h->z.p, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr,
                h->vxd.p, h->vyd.p, h->vzd.p, h->xr.p, h->yr.p, h->zr.p, h->flags.p, h->t_death.p, h->t_arr.p, h->mom_partials.p);
        } else if (h->hilo()) {
            k_moments_partial<float, true><<<h->n_mom_items, 256, 0, s>>>(
                h->mom_items.p, nullptr, nullptr, nullptr, h->xh.p, h->xl.p, h->yh.p, h->yl.p, h->zh.p, h->zl.p,
                h->vxf.p, h->vyf.p, h->vzf.p, h->xr.p, h->yr.p, h->zr.p, h->flags.p, h->t_death.p, h->t_arr.p, h->mom_partials.p);
        } else {
            k_moments_partial<float, false><<<h->n_mom_items, 256, 0, s>>>(
                h->mom_items.p, h->x.p, h->y.p, h->z.p, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr,
                h->vxf.p, h->vyf.p, h->vzf.p, h->xr.p, h->yr.p, h->zr.p, h->flags.p, h->t_death.p, h->t_arr.p, h->mom_partials.p);
        }
        ICB_CUDA(cudaGetLastError());
    }
    k_moments_final<<<ne, 32, 0, s>>>(h->mom_partials.p, h->mom_item_off.p, ne, h->mom_out.p);
    ICB_CUDA(cudaGetLastError());
    ICB_CUDA(cudaMemcpyAsync(out, h->mom_out.p, static_cast<size_t>(ne) * ICB_N_MOMENTS * sizeof(double), cudaMemcpyDeviceToHost, s));
    ICB_CUDA(cudaStreamSynchronize(s));
    return ICB_OK;
}

int icb_mark_reference(icb_handle* h) {
    if (int r = check_handle(h)) return r;
    if (h->n == 0) return fail(ICB_ERR_STATE, "no ions uploaded");
    cudaStream_t s = h->stream;
    const uint64_t n = h->n;
    if (h->hilo()) {
        const unsigned g = grid_for(n, 256);
        k_from_hilo<<<g, 256, 0, s>>>(h->xh.p, h->xl.p, h->xr.p, n);
        k_from_hilo<<<g, 256, 0, s>>>(h->yh.p, h->yl.p, h->yr.p, n);
        k_from_hilo<<<g, 256, 0, s>>>(h->zh.p, h->zl.p, h->zr.p, n);
        ICB_CUDA(cudaGetLastError());
    } else {
        ICB_CUDA(cudaMemcpyAsync(h->xr.p, h->x.p, n * sizeof(double), cudaMemcpyDeviceToDevice, s));
        ICB_CUDA(cudaMemcpyAsync(h->yr.p, h->y.p, n * sizeof(double), cudaMemcpyDeviceToDevice, s));
        ICB_CUDA(cudaMemcpyAsync(h->zr.p, h->z.p, n * sizeof(double), cudaMemcpyDeviceToDevice, s));
    }
    return ICB_OK;
}

}  // extern "C"
