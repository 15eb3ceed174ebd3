// icb_p3m.cu — space-charge field of the ion cloud (ISpaceChargeModel,
// ISpaceChargeModel.h:22-46), solved once per step before the push.
//
// Two solvers share one pipeline:
//   bin     ions -> mesh base cell key (CIC cell of the lower corner)
//   sort    (key, ion) pairs, stable radix sort (CUB)
//   bounds  first sorted slot of every cell key (binary search)
//   deposit every mesh node gathers the CIC charge of the ions in the eight
//           cells around it, in a fixed order (deterministic, no atomics)
//   solve   isolated P3M: zero-padded (2n)^3 FFT convolution with the
//           transformed long-range field kernel (three inverse FFTs, one per
//           field component); periodic PM (the reference's solver as it is,
//           GPUSpaceChargeP3M.cu:36-339): periodic Poisson solve, 1/N scale,
//           central differences
//   gather  per ion (in cell order): CIC interpolation of the mesh field,
//           plus, for P3M, the particle-particle correction over the ions in
//           the cells within the cutoff
// All arithmetic is FP64; the periodic solver keeps the reference's float
// CIC weights and float field output.
#include <cuda_runtime.h>
#include <cufft.h>

#include <cub/device/device_radix_sort.cuh>
#include <cub/device/device_scan.cuh>

#include <algorithm>
#include <climits>
#include <cmath>
#include <cstdio>
#include <memory>
#include <string>
#include <vector>

#include "../../include/icarion_b200.h"
#include "icb_internal.h"

namespace icb {

namespace {

constexpr double kCoulomb = 8.987551787e9;     // utils/constants.h:20
constexpr double kEps0 = 8.854187817e-12;      // utils/constants.h:19
constexpr double kPi = 3.14159265358979323846;

struct MeshGeom {
    int n0, n1, n2;          // mesh nodes
    int m0, m1, m2;          // FFT grid
    double lo0, lo1, lo2;
    double ih0, ih1, ih2;    // grid coordinate scale (1/h, or n/extent for the periodic solver)
    uint32_t ncell;          // n0*n1*n2 (also the key of excluded ions)
};

__device__ __forceinline__ bool grid_coords(const MeshGeom& g, double x, double y, double z, double f[3]) {
    f[0] = (x - g.lo0) * g.ih0;
    f[1] = (y - g.lo1) * g.ih1;
    f[2] = (z - g.lo2) * g.ih2;
    // false for NaN as well
    return f[0] >= 0.0 && f[0] < g.n0 - 1 && f[1] >= 0.0 && f[1] < g.n1 - 1 && f[2] >= 0.0 && f[2] < g.n2 - 1;
}

// Slots [0, n_own) are this handle's ions; slots n_own + j the peers' ions j
// (other devices' ions in the same solve: position, charge; a peer takes
// part when its charge is nonzero and j is outside the skip range).
struct PeerIons {
    const double4* xyzq = nullptr;
    uint32_t n = 0, skip_b = 0, skip_n = 0;
};

__global__ void k_sc_bin(MeshGeom g, const double* __restrict__ x, const double* __restrict__ y,
                         const double* __restrict__ z, const uint8_t* __restrict__ flags, uint32_t n_own,
                         PeerIons peers, int all_ions, uint32_t* __restrict__ keys, uint32_t* __restrict__ vals) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n_own + peers.n) return;
    uint32_t key = g.ncell;
    bool use;
    double px, py, pz;
    if (i < n_own) {
        use = all_ions || ((flags[i] & 3u) == 3u);   // active and born
        px = x[i]; py = y[i]; pz = z[i];
    } else {
        const uint32_t j = i - n_own;
        const double4 v = peers.xyzq[j];
        use = v.w != 0.0 && (j < peers.skip_b || j - peers.skip_b >= peers.skip_n);
        px = v.x; py = v.y; pz = v.z;
    }
    double f[3];
    if (use && grid_coords(g, px, py, pz, f)) {
        const int c0 = static_cast<int>(f[0]), c1 = static_cast<int>(f[1]), c2 = static_cast<int>(f[2]);
        key = (static_cast<uint32_t>(c0) * g.n1 + static_cast<uint32_t>(c1)) * g.n2 + static_cast<uint32_t>(c2);
    }
    keys[i] = key;
    vals[i] = i;
}

// start[c] = first sorted slot whose key is >= c, for c in [0, ncell]: one
// binary search per group of four cells, then a forward scan over the keys
// (a cell holds a few ions).
__global__ void k_sc_cell_start(const uint32_t* __restrict__ keys, uint32_t n, uint32_t ncell,
                                uint32_t* __restrict__ start) {
    const uint32_t c0 = 4u * (blockIdx.x * blockDim.x + threadIdx.x);
    if (c0 > ncell) return;
    uint32_t lo = 0, hi = n;
    while (lo < hi) {
        const uint32_t mid = lo + ((hi - lo) >> 1);
        if (keys[mid] < c0) lo = mid + 1; else hi = mid;
    }
    for (uint32_t c = c0; c < c0 + 4u && c <= ncell; ++c) {
        while (lo < n && keys[lo] < c) ++lo;
        start[c] = lo;
    }
}

// Positions and charges in sorted (cell) order: the deposit and the
// particle-particle loops then read contiguous memory.
// A float copy (position relative to the mesh origin, Coulomb constant times
// the charge) serves the particle-particle loop: per slot (x, y, z, kq) as
// the FP64 loop's distance prefilter, or, for the float loop (`pairs`), per
// slot pair k = s / 2 as two float4 {x0, x1, y0, y1}, {z0, z1, kq0, kq1}:
// the packed (two-lane) FP32 instructions then take each pair's values as
// loaded.
__global__ void k_sc_permute(MeshGeom g, const double* __restrict__ x, const double* __restrict__ y,
                             const double* __restrict__ z, const double* __restrict__ q,
                             const uint32_t* __restrict__ vals, uint32_t n, uint32_t n_own, PeerIons peers,
                             int pairs, double4* __restrict__ ps, float4* __restrict__ pf) {
    const uint32_t s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= n) return;
    const uint32_t j = vals[s];
    const double4 v = j < n_own ? make_double4(x[j], y[j], z[j], q[j]) : peers.xyzq[j - n_own];
    ps[s] = v;
    const float fx = static_cast<float>(v.x - g.lo0), fy = static_cast<float>(v.y - g.lo1);
    const float fz = static_cast<float>(v.z - g.lo2), fq = static_cast<float>(kCoulomb * v.w);
    if (pairs) {
        float* b = reinterpret_cast<float*>(pf) + 8u * (s >> 1) + (s & 1u);
        b[0] = fx; b[2] = fy; b[4] = fz; b[6] = fq;
    } else {
        pf[s] = make_float4(fx, fy, fz, fq);
    }
}

// Sorted slots of this handle's own ions, in sorted order: a flag per slot,
// its exclusive scan, then the scatter of the flagged slots.
__global__ void k_sc_own_flag(const uint32_t* __restrict__ vals, uint32_t n, uint32_t n_own,
                              uint32_t* __restrict__ flag) {
    const uint32_t s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s < n) flag[s] = vals[s] < n_own ? 1u : 0u;
}
__global__ void k_sc_own_scatter(const uint32_t* __restrict__ vals, const uint32_t* __restrict__ pos, uint32_t n,
                                 uint32_t n_own, uint32_t* __restrict__ slots) {
    const uint32_t s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s < n && vals[s] < n_own) slots[pos[s]] = s;
}

// This handle's ions as a peer list for other devices' solves: active, born
// ions keep position and charge; the rest get charge 0 (they take no part).
__global__ void k_sc_export(const double* __restrict__ x, const double* __restrict__ y, const double* __restrict__ z,
                            const double* __restrict__ q, const uint8_t* __restrict__ flags, uint64_t n,
                            double4* __restrict__ out) {
    const uint64_t i = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const bool use = (flags[i] & 3u) == 3u;
    out[i] = use ? make_double4(x[i], y[i], z[i], q[i]) : make_double4(0.0, 0.0, 0.0, 0.0);
}

// CIC weight of corner (ox, oy, oz) of a cell for fractions fr (taken left
// to right: x, y, z).
template <class W>
__device__ __forceinline__ W cic_w(int ox, int oy, int oz, W fx, W fy, W fz) {
    const W one = W(1);
    return (ox ? fx : one - fx) * (oy ? fy : one - fy) * (oz ? fz : one - fz);
}

// Charge per mesh node (C), written into the FFT grid (whose nodes outside
// the mesh were zeroed before).  One thread per mesh node.
template <bool REF_WEIGHTS, class T>
__global__ void k_sc_deposit(MeshGeom g, const double4* __restrict__ ps, const uint32_t* __restrict__ start,
                             T* __restrict__ rho) {
    const size_t total = static_cast<size_t>(g.n0) * g.n1 * g.n2;
    const size_t idx = static_cast<size_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (idx >= total) return;
    const int c = static_cast<int>(idx % g.n2);
    const size_t t = idx / g.n2;
    const int b = static_cast<int>(t % g.n1);
    const int a = static_cast<int>(t / g.n1);
    // cells (ci, cj, ck) with ck = c - 1, c are adjacent keys: one slot range
    // per (ci, cj) column, each ion's ck taken from its position as k_sc_bin
    // took it (the same sums in the same order as cell by cell)
    const int kz0 = max(c - 1, 0), kz1 = min(c, g.n2 - 2);
    double acc = 0.0;
    for (int ci = a - 1; ci <= a; ++ci) {
        if (ci < 0 || ci > g.n0 - 2) continue;
        for (int cj = b - 1; cj <= b; ++cj) {
            if (cj < 0 || cj > g.n1 - 2 || kz0 > kz1) continue;
            const uint32_t row = (static_cast<uint32_t>(ci) * g.n1 + static_cast<uint32_t>(cj)) * g.n2;
            const uint32_t s1 = start[row + static_cast<uint32_t>(kz1) + 1u];
            for (uint32_t s = start[row + static_cast<uint32_t>(kz0)]; s < s1; ++s) {
                const double4 pj = ps[s];
                const double gz = (pj.z - g.lo2) * g.ih2;
                const int ck = static_cast<int>(gz);
                const double fx = (pj.x - g.lo0) * g.ih0 - ci;
                const double fy = (pj.y - g.lo1) * g.ih1 - cj;
                const double fz = gz - ck;
                double w;
                if (REF_WEIGHTS) {
                    w = static_cast<double>(cic_w<float>(a - ci, b - cj, c - ck, static_cast<float>(fx),
                                                         static_cast<float>(fy), static_cast<float>(fz)));
                } else {
                    w = cic_w<double>(a - ci, b - cj, c - ck, fx, fy, fz);
                }
                acc += w * pj.w;
            }
        }
    }
    rho[(static_cast<size_t>(a) * g.m1 + static_cast<size_t>(b)) * g.m2 + static_cast<size_t>(c)] = static_cast<T>(acc);
}

// out_c = a * b_c (complex) for the three field components, n entries each
template <class CT>
__global__ void k_sc_cmul3(const CT* __restrict__ a, const CT* __restrict__ b0, const CT* __restrict__ b1,
                           const CT* __restrict__ b2, CT* __restrict__ out, size_t n) {
    const size_t i = static_cast<size_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const CT u = a[i];
    const CT* bs[3] = {b0, b1, b2};
#pragma unroll
    for (int c = 0; c < 3; ++c) {
        const CT v = bs[c][i];
        CT r;
        r.x = u.x * v.x - u.y * v.y;
        r.y = u.x * v.y + u.y * v.x;
        out[c * n + i] = r;
    }
}

// Single-precision mesh of the isolated solver.  Field component c's
// sampled kernel is real, odd along axis c and even along the other two
// (k_sc_green), so its transform is imaginary, odd in k_c and even in the
// other wave numbers.  Only the imaginary part on the quadrant
// kx <= m0/2, ky <= m1/2 (all kz of the half spectrum) is kept: 1/8 of the
// complex array, small enough to stay in L2 while the product streams.
struct FoldGeom {
    int hx, hy, hz;          // m0/2 + 1, m1/2 + 1, m2/2 + 1
    size_t n;                // hx * hy * hz
};
__host__ __device__ inline FoldGeom fold_geom(const MeshGeom& g) {
    FoldGeom f;
    f.hx = g.m0 / 2 + 1; f.hy = g.m1 / 2 + 1; f.hz = g.m2 / 2 + 1;
    f.n = static_cast<size_t>(f.hx) * f.hy * f.hz;
    return f;
}

// Layout [kx][ky][kz], or with `kx_inner` [ky][kz][kx] (the fused x pass
// reads a column's kx run contiguously).
__global__ void k_sc_fold(MeshGeom g, const cufftDoubleComplex* __restrict__ gh, int kx_inner,
                          float* __restrict__ out) {
    const FoldGeom f = fold_geom(g);
    const size_t idx = static_cast<size_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (idx >= f.n) return;
    const int kz = static_cast<int>(idx % f.hz);
    const size_t t = idx / f.hz;
    const int ky = static_cast<int>(t % f.hy);
    const int kx = static_cast<int>(t / f.hy);
    const size_t o = kx_inner ? (static_cast<size_t>(ky) * f.hz + kz) * f.hx + kx : idx;
    out[o] = static_cast<float>(gh[(static_cast<size_t>(kx) * g.m1 + ky) * f.hz + kz].y);
}

// out_c = rho_hat * (i G_c) for the three components.  One thread per
// folded point: it reads G_c once and serves the point's mirrors
// (kx, m0 - kx) x (ky, m1 - ky), flipping G_0 at m0 - kx and G_1 at
// m1 - ky (kx = 0 or m0/2, and likewise ky, are their own mirrors).
__global__ void k_sc_cmul_fold(MeshGeom g, const cufftComplex* __restrict__ a, const float* __restrict__ gf,
                               cufftComplex* __restrict__ out) {
    const FoldGeom f = fold_geom(g);
    const size_t idx = static_cast<size_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (idx >= f.n) return;
    const int kz = static_cast<int>(idx % f.hz);
    const size_t t = idx / f.hz;
    const int ky = static_cast<int>(t % f.hy);
    const int kx = static_cast<int>(t / f.hy);
    const float G0 = gf[idx], G1 = gf[f.n + idx], G2 = gf[2 * f.n + idx];
    const size_t plane = static_cast<size_t>(g.m1) * f.hz;
    const size_t n = static_cast<size_t>(g.m0) * plane;
    const int nx = (kx == 0 || 2 * kx == g.m0) ? 1 : 2;
    const int ny = (ky == 0 || 2 * ky == g.m1) ? 1 : 2;
    for (int mx = 0; mx < nx; ++mx) {
        const size_t X = static_cast<size_t>(mx ? g.m0 - kx : kx);
        const float g0 = mx ? -G0 : G0;
        for (int my = 0; my < ny; ++my) {
            const size_t Y = static_cast<size_t>(my ? g.m1 - ky : ky);
            const float gc[3] = {g0, my ? -G1 : G1, G2};
            const size_t o = X * plane + Y * f.hz + kz;
            const cufftComplex u = a[o];
#pragma unroll
            for (int c = 0; c < 3; ++c) out[c * n + o] = make_cuComplex(-u.y * gc[c], u.x * gc[c]);
        }
    }
}

// ---------------------------------------------------------------------------
// Fused x pass of the single-precision mesh for a padded x length of 256 (a
// 128-node mesh axis).  Per (ky, kz) column of the 2D-transformed mesh
// planes: the forward 256-point transform along x (inputs x >= 128 are the
// zero padding), the products with i G_c of the three field components,
// and their inverse transforms, keeping the outputs x < 128 (the mesh
// planes the gather reads).  The unfused path's three whole spectra are
// never written or read back.  256 = 16 x 16: a block of 256 threads takes
// 16 columns, 16 threads a column, each thread 16 points in registers; a
// transform is two 16-point DFTs with the 256-point twiddles between them
// and one transpose through shared memory (rows of 17 against bank
// conflicts; 273 float2 a column keeps the column-major staging
// conflict-free too).
constexpr int kXLen = 256;
constexpr int kXCols = 16;
constexpr int kXStride = 273;

__device__ __forceinline__ float2 cmulf(float2 a, float2 b) {
    return make_float2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}

// 4-point DFT in place, y_k = sum_n a_n w^(n k), w = -i (forward) or +i.
template <bool INV>
__device__ __forceinline__ void dft4(float2& a0, float2& a1, float2& a2, float2& a3) {
    const float2 s02 = make_float2(a0.x + a2.x, a0.y + a2.y), d02 = make_float2(a0.x - a2.x, a0.y - a2.y);
    const float2 s13 = make_float2(a1.x + a3.x, a1.y + a3.y), d13 = make_float2(a1.x - a3.x, a1.y - a3.y);
    const float2 r = INV ? make_float2(-d13.y, d13.x) : make_float2(d13.y, -d13.x);   // w * d13
    a0 = make_float2(s02.x + s13.x, s02.y + s13.y);
    a1 = make_float2(d02.x + r.x, d02.y + r.y);
    a2 = make_float2(s02.x - s13.x, s02.y - s13.y);
    a3 = make_float2(d02.x - r.x, d02.y - r.y);
}

// exp(-+2 pi i m / 16) for the exponents a 4 x 4 split uses (m = n2 k1)
template <bool INV>
__device__ __forceinline__ float2 w16(int m) {
    constexpr float c1 = 0.923879532511286756f, s1 = 0.382683432365089772f, r2 = 0.707106781186547524f;
    float c = 1.f, sn = 0.f;
    switch (m) {
        case 1: c = c1; sn = s1; break;
        case 2: c = r2; sn = r2; break;
        case 3: c = s1; sn = c1; break;
        case 4: c = 0.f; sn = 1.f; break;
        case 6: c = -r2; sn = r2; break;
        case 9: c = -c1; sn = -s1; break;
        default: break;
    }
    return make_float2(c, INV ? sn : -sn);
}

// 16-point DFT in registers, v_k = sum_n v_n w^(n k), w = exp(-+2 pi i/16):
// n = 4 n1 + n2, k = k1 + 4 k2; 4-point DFTs over n1, twiddles w^(n2 k1),
// 4-point DFTs over n2, then natural order.
template <bool INV>
__device__ __forceinline__ void dft16(float2 (&v)[16]) {
#pragma unroll
    for (int n2 = 0; n2 < 4; ++n2) dft4<INV>(v[n2], v[4 + n2], v[8 + n2], v[12 + n2]);
#pragma unroll
    for (int n2 = 1; n2 < 4; ++n2) {
#pragma unroll
        for (int k1 = 1; k1 < 4; ++k1) v[4 * k1 + n2] = cmulf(v[4 * k1 + n2], w16<INV>(n2 * k1));
    }
#pragma unroll
    for (int k1 = 0; k1 < 4; ++k1) dft4<INV>(v[4 * k1], v[4 * k1 + 1], v[4 * k1 + 2], v[4 * k1 + 3]);
    float2 t[16];
#pragma unroll
    for (int k1 = 0; k1 < 4; ++k1) {
#pragma unroll
        for (int k2 = 0; k2 < 4; ++k2) t[k1 + 4 * k2] = v[4 * k1 + k2];
    }
#pragma unroll
    for (int k = 0; k < 16; ++k) v[k] = t[k];
}

// in: the mesh planes x < 128 of the 2D-transformed charge, [x][ky][kz];
// gf: the folded kernels, [c][ky][kz][kx] (k_sc_fold with kx_inner);
// out: component c's planes x < 128 after the x pass, at c * 128 * P;
// tw: exp(-2 pi i m / 256), m < 256.
__global__ void __launch_bounds__(256, 3) k_sc_xconv(MeshGeom g, const float2* __restrict__ in,
                                                  const float* __restrict__ gf, const float2* __restrict__ tw,
                                                  float2* __restrict__ out) {
    __shared__ float2 buf[kXCols * kXStride];
    __shared__ float2 w[kXLen];
    const FoldGeom f = fold_geom(g);
    const uint32_t P = static_cast<uint32_t>(g.m1) * static_cast<uint32_t>(f.hz);    // (ky, kz) columns
    const uint32_t j0 = blockIdx.x * kXCols;
    const int col = threadIdx.x >> 4, t = threadIdx.x & 15;
    w[threadIdx.x] = tw[threadIdx.x];
    for (int e = threadIdx.x; e < (kXLen / 2) * kXCols; e += blockDim.x) {
        const int x = e >> 4, c = e & 15;
        const uint32_t j = j0 + c;
        buf[c * kXStride + x] = j < P ? in[static_cast<size_t>(x) * P + j] : make_float2(0.f, 0.f);
    }
    __syncthreads();
    float2* bc = buf + col * kXStride;
    float2 v[16];
    // forward: x = 16 x1 + t, k = k1 + 16 k2
#pragma unroll
    for (int x1 = 0; x1 < 16; ++x1) v[x1] = x1 < 8 ? bc[16 * x1 + t] : make_float2(0.f, 0.f);
    __syncthreads();
    dft16<false>(v);
#pragma unroll
    for (int k1 = 0; k1 < 16; ++k1) bc[t * 17 + k1] = cmulf(v[k1], w[(t * k1) & 255]);
    __syncthreads();
#pragma unroll
    for (int x2 = 0; x2 < 16; ++x2) v[x2] = bc[x2 * 17 + t];
    dft16<false>(v);
    float2 X[16];                                   // X[k2] = spectrum at kx = t + 16 k2
#pragma unroll
    for (int k2 = 0; k2 < 16; ++k2) X[k2] = v[k2];
    const uint32_t j = j0 + col;
    const bool live = j < P;
    const int ky = live ? static_cast<int>(j / f.hz) : 0, kz = live ? static_cast<int>(j % f.hz) : 0;
    const int kyf = min(ky, g.m1 - ky);
    const float sy = 2 * ky > g.m1 ? -1.f : 1.f;
    for (int c = 0; c < 3; ++c) {
        // kernel values in [ky][kz][kx] order: a column's kx run is contiguous
        const float* gc = gf + c * f.n + (static_cast<size_t>(kyf) * f.hz + kz) * f.hx;
#pragma unroll
        for (int k2 = 0; k2 < 16; ++k2) {
            const int kx = t + 16 * k2;
            const int kxf = min(kx, kXLen - kx);
            float G = live ? gc[kxf] : 0.f;
            if (c == 0 && kx > kXLen / 2) G = -G;
            if (c == 1) G *= sy;
            v[k2] = make_float2(-G * X[k2].y, G * X[k2].x);
        }
        // inverse: k = t + 16 k2, x = r + 16 q; only q < 8 is kept
        dft16<true>(v);
        __syncthreads();
#pragma unroll
        for (int r = 0; r < 16; ++r) {
            const float2 wr = w[(r * t) & 255];
            bc[r * 17 + t] = cmulf(v[r], make_float2(wr.x, -wr.y));
        }
        __syncthreads();
#pragma unroll
        for (int k1 = 0; k1 < 16; ++k1) v[k1] = bc[t * 17 + k1];
        dft16<true>(v);
        __syncthreads();
#pragma unroll
        for (int q = 0; q < 8; ++q) bc[t + 16 * q] = v[q];
        __syncthreads();
        float2* oc = out + static_cast<size_t>(c) * (kXLen / 2) * P;
        for (int e = threadIdx.x; e < (kXLen / 2) * kXCols; e += blockDim.x) {
            const int x = e >> 4, cc = e & 15;
            if (j0 + cc < P) oc[static_cast<size_t>(x) * P + j0 + cc] = buf[cc * kXStride + x];
        }
    }
}

__device__ __forceinline__ double e_long(double r, double alpha) {
    // long-range part of a unit charge's field / Coulomb constant:
    // erf(a r)/r^2 - (2a/sqrt(pi)) exp(-a^2 r^2)/r
    const double ar = alpha * r;
    return erf(ar) / (r * r) - (2.0 * alpha / sqrt(kPi)) * exp(-ar * ar) / r;
}

// Component `comp` of the sampled long-range field of a unit charge on the
// zero-padded grid: displacement index s wrapped to (-n, n); s == n is never
// reached by mesh data and is 0, as is the origin.
__global__ void k_sc_green(MeshGeom g, double h0, double h1, double h2, double alpha, int comp,
                           double* __restrict__ out) {
    const size_t total = static_cast<size_t>(g.m0) * g.m1 * g.m2;
    const size_t idx = static_cast<size_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (idx >= total) return;
    const int c = static_cast<int>(idx % g.m2);
    const size_t t = idx / g.m2;
    const int b = static_cast<int>(t % g.m1);
    const int a = static_cast<int>(t / g.m1);
    double v = 0.0;
    if (a != g.n0 && b != g.n1 && c != g.n2) {
        const double dx = (a < g.n0 ? a : a - g.m0) * h0;
        const double dy = (b < g.n1 ? b : b - g.m1) * h1;
        const double dz = (c < g.n2 ? c : c - g.m2) * h2;
        const double r2 = dx * dx + dy * dy + dz * dz;
        if (r2 > 0.0) {
            const double r = sqrt(r2);
            const double f = kCoulomb * e_long(r, alpha) / r;
            v = f * (comp == 0 ? dx : (comp == 1 ? dy : dz));
        }
    }
    out[idx] = v;
}

// Scale a transformed kernel by 1 / (grid size): cuFFT's inverse is
// unnormalised.
__global__ void k_sc_normalize(MeshGeom g, cufftDoubleComplex* __restrict__ gh) {
    const size_t total = static_cast<size_t>(g.m0) * g.m1 * (g.m2 / 2 + 1);
    const size_t idx = static_cast<size_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (idx >= total) return;
    const double scale = 1.0 / (static_cast<double>(g.m0) * g.m1 * g.m2);
    gh[idx].x *= scale;
    gh[idx].y *= scale;
}

// The reference's Fourier-space Poisson step (GPUSpaceChargeP3M.cu:114-161):
// phi_hat = rho_hat / (eps0 k^2 V), k = 0 -> 0, its z length (nz/2+1) 2 dz.
__global__ void k_sc_poisson_ref(MeshGeom g, double dx, double dy, double dz, cufftDoubleComplex* __restrict__ rh) {
    const int nx = g.n0, ny = g.n1, nz_half = g.n2 / 2 + 1;
    const int total = nx * ny * nz_half;
    const int mode_idx = blockIdx.x * blockDim.x + threadIdx.x;
    if (mode_idx >= total) return;
    const int i = mode_idx / (ny * nz_half);
    const int j = (mode_idx % (ny * nz_half)) / nz_half;
    const int k = mode_idx % nz_half;
    const double Lx = nx * dx, Ly = ny * dy, Lz = nz_half * 2 * dz;
    const double kx = (i < nx / 2) ? (2.0 * kPi * i / Lx) : (2.0 * kPi * (i - nx) / Lx);
    const double ky = (j < ny / 2) ? (2.0 * kPi * j / Ly) : (2.0 * kPi * (j - ny) / Ly);
    const double kz = 2.0 * kPi * k / Lz;
    const double k2 = kx * kx + ky * ky + kz * kz;
    if (k2 < 1e-10) {
        rh[mode_idx].x = 0.0;
        rh[mode_idx].y = 0.0;
        return;
    }
    const double scale = 1.0 / (kEps0 * k2 * (dx * dy * dz));
    rh[mode_idx].x = rh[mode_idx].x * scale;
    rh[mode_idx].y = rh[mode_idx].y * scale;
}

// E = -grad(phi * s) by central differences, one-sided at the edges
// (GPUSpaceChargeP3M.cu:176-248).
__global__ void k_sc_efield_ref(MeshGeom g, double dx, double dy, double dz, double s, const double* __restrict__ phi,
                                double* __restrict__ ex, double* __restrict__ ey, double* __restrict__ ez) {
    const int nx = g.n0, ny = g.n1, nz = g.n2;
    const int total = nx * ny * nz;
    const int cell = blockIdx.x * blockDim.x + threadIdx.x;
    if (cell >= total) return;
    const int i = cell / (ny * nz);
    const int j = (cell % (ny * nz)) / nz;
    const int k = cell % nz;
    const int sy = nz, sx = ny * nz;
    auto P = [&](int a, int b, int c) { return phi[a * sx + b * sy + c] * s; };
    if (i == 0) ex[cell] = -(P(i + 1, j, k) - P(i, j, k)) / dx;
    else if (i == nx - 1) ex[cell] = -(P(i, j, k) - P(i - 1, j, k)) / dx;
    else ex[cell] = -(P(i + 1, j, k) - P(i - 1, j, k)) / (2.0 * dx);
    if (j == 0) ey[cell] = -(P(i, j + 1, k) - P(i, j, k)) / dy;
    else if (j == ny - 1) ey[cell] = -(P(i, j, k) - P(i, j - 1, k)) / dy;
    else ey[cell] = -(P(i, j + 1, k) - P(i, j - 1, k)) / (2.0 * dy);
    if (k == 0) ez[cell] = -(P(i, j, k + 1) - P(i, j, k)) / dz;
    else if (k == nz - 1) ez[cell] = -(P(i, j, k) - P(i, j, k - 1)) / dz;
    else ez[cell] = -(P(i, j, k + 1) - P(i, j, k - 1)) / (2.0 * dz);
}

struct PPParams {
    int on;
    int r0, r1, r2;          // neighbour cell reach per axis
    double rc2, alpha, eps2, min_d2;
    float rc2_pre;           // float prefilter bound, slightly above rc^2
    double inv_dr;           // table intervals per metre
    const double* table;     // L(r) at r = k / inv_dr, k = 0..kPPTable
    // float particle-particle arithmetic (the float forms): bounds in float
    int use_float;
    float rc2f, eps2f, min_d2f, inv_drf;
    // the float loop's long-range term as a polynomial when it is accurate
    // enough (sc_create checks): -L(r)/r^3 = sum_k pc[k] u^k, u = r^2 pu_s - 1
    int poly;
    float pu_s;
    float pc[11];
};
constexpr int kPPPoly = 10;     // degree of that polynomial

// Particle-particle table: L(r) = r^2 E_long(r) / k = erf(a r) - (2 a r /
// sqrt(pi)) exp(-a^2 r^2) on kPPTable equal intervals of [0, r_c], linearly
// interpolated (relative error ~ (a r_c / kPPTable)^2 / 8 ~ 3e-8 at a r_c = 2).
constexpr int kPPTable = 4096;

// Field of one ion: CIC interpolation of the mesh field (+ particle-
// particle correction).  Thread tt handles the ion in sorted slot tt (or
// slots[tt]).
template <bool REF_WEIGHTS, class GT, bool POLY>
__device__ __forceinline__ void sc_gather_ion(uint32_t tt, const MeshGeom& g, const PPParams& pp,
                            const double4* __restrict__ ps, const float4* __restrict__ pf,
                            const uint32_t* __restrict__ keys, const uint32_t* __restrict__ vals,
                            const uint32_t* __restrict__ start, uint32_t n, const uint32_t* __restrict__ slots,
                            const GT* __restrict__ gx, const GT* __restrict__ gy, const GT* __restrict__ gz,
                            double* __restrict__ ex, double* __restrict__ ey, double* __restrict__ ez,
                            const double* tab, const float* tabf) {
    // Every lane of a warp reaches the particle-particle loops (they use
    // warp-wide ranges); lanes without an ion inside the mesh take part with
    // empty ranges.
    // thread t takes sorted slot t, or slots[t] (this handle's ions among
    // peers' ions: n counts the own ions then)
    const bool in_range = tt < n;
    const uint32_t s = in_range ? (slots ? slots[tt] : tt) : 0u;
    const uint32_t i = in_range ? vals[s] : 0u;
    const uint32_t key = in_range ? keys[s] : g.ncell;
    const bool act = key < g.ncell;
    if (!REF_WEIGHTS && pp.on && pp.use_float && __all_sync(0xffffffffu, !act)) {
        if (in_range) { ex[i] = 0.0; ey[i] = 0.0; ez[i] = 0.0; }
        return;
    }
    if (!act && (REF_WEIGHTS || !pp.on || !pp.use_float)) {
        if (in_range) { ex[i] = 0.0; ey[i] = 0.0; ez[i] = 0.0; }
        return;
    }
    const uint32_t keyc = act ? key : 0u;
    const int ck = static_cast<int>(keyc % g.n2);
    const uint32_t t = keyc / g.n2;
    const int cj = static_cast<int>(t % g.n1);
    const int ci = static_cast<int>(t / g.n1);
    double E[3] = {0.0, 0.0, 0.0};
    const double4 pi4 = act ? ps[s] : make_double4(0.0, 0.0, 0.0, 0.0);
    const double xi = pi4.x, yi = pi4.y, zi = pi4.z;
    if (act) {
        const double fx = (xi - g.lo0) * g.ih0 - ci;
        const double fy = (yi - g.lo1) * g.ih1 - cj;
        const double fz = (zi - g.lo2) * g.ih2 - ck;
        const GT* grid[3] = {gx, gy, gz};
        // corners in the reference's order w000, w100, w010, w110, w001, ... (x fastest)
        for (int oz = 0; oz < 2; ++oz) {
            for (int oy = 0; oy < 2; ++oy) {
                for (int ox = 0; ox < 2; ++ox) {
                    double w;
                    if (REF_WEIGHTS) {
                        w = static_cast<double>(cic_w<float>(ox, oy, oz, static_cast<float>(fx), static_cast<float>(fy),
                                                             static_cast<float>(fz)));
                    } else {
                        w = cic_w<double>(ox, oy, oz, fx, fy, fz);
                    }
                    const size_t node = (static_cast<size_t>(ci + ox) * g.m1 + static_cast<size_t>(cj + oy)) * g.m2 +
                                        static_cast<size_t>(ck + oz);
#pragma unroll
                    for (int c = 0; c < 3; ++c) E[c] += w * static_cast<double>(grid[c][node]);
                }
            }
        }
        if (REF_WEIGHTS) {
#pragma unroll
            for (int c = 0; c < 3; ++c) E[c] = static_cast<double>(static_cast<float>(E[c]));
        }
    }
    if (!REF_WEIGHTS && pp.on) {
        const int x0 = max(ci - pp.r0, 0), x1 = min(ci + pp.r0, g.n0 - 2);
        const int y0 = max(cj - pp.r1, 0), y1 = min(cj + pp.r1, g.n1 - 2);
        const int z0 = max(ck - pp.r2, 0), z1 = min(ck + pp.r2, g.n2 - 2);
        if (pp.use_float) {
            // float arithmetic on positions relative to the mesh origin,
            // partners read as slot pairs (k_sc_permute) and evaluated two
            // at a time on the packed FP32 pipe (sm_100 fma/add/mul .f32x2:
            // one instruction for both).
            // Each (cx, cy) column contributes the cells whose z interval
            // reaches within r_c of the ion given the column's distance in x
            // and y (lower bounds, padded for rounding).  The warp walks the
            // union of its lanes' slot ranges together (one broadcast load
            // per pair) only when that union is barely longer than the
            // longest range; otherwise each lane walks its own range (the
            // warp pays the longest, with nearby loads): over the sorted
            // FT-ICR cloud this evaluates ~1.6 pairs per useful one where
            // walking unions costs ~2.2.  Pairs outside a lane's range or
            // outside (min_d, r_c) add exactly nothing (the ion itself is at
            // distance 0 < min_d), so the sums equal a walk over every pair
            // of the cells within reach.
            const unsigned full = 0xffffffffu;
            float fxi = 0.f, fyi = 0.f, fzi = 0.f;
            if (act) {
                const float* b = reinterpret_cast<const float*>(pf) + 8u * (s >> 1) + (s & 1u);
                fxi = b[0]; fyi = b[2]; fzi = b[4];
            }
            const float h0 = static_cast<float>(1.0 / g.ih0), h1 = static_cast<float>(1.0 / g.ih1);
            const float ih2 = static_cast<float>(g.ih2);
            const float rcpad = pp.rc2f * 1.0001f;
            const float zpad = 1e-4f * static_cast<float>(1.0 / g.ih2);
            const float2 m1 = make_float2(-1.f, -1.f);
            const float2 FX = make_float2(fxi, fxi), FY = make_float2(fyi, fyi), FZ = make_float2(fzi, fzi);
            const float2 INV = make_float2(pp.inv_drf, pp.inv_drf), EPS = make_float2(pp.eps2f, pp.eps2f);
            const float2 US = make_float2(pp.pu_s, pp.pu_s);
            float2 E2x = make_float2(0.f, 0.f), E2y = E2x, E2z = E2x;
            // partners 2k and 2k + 1 (ta, tb: inside the lane's range)
            auto pair2 = [&](uint32_t k, bool ta, bool tb) {
                const float4 xy = pf[2u * k], zq = pf[2u * k + 1u];
                const float2 dX = __ffma2_rn(make_float2(xy.x, xy.y), m1, FX);
                const float2 dY = __ffma2_rn(make_float2(xy.z, xy.w), m1, FY);
                const float2 dZ = __ffma2_rn(make_float2(zq.x, zq.y), m1, FZ);
                const float2 r2 = __ffma2_rn(dZ, dZ, __ffma2_rn(dY, dY, __fmul2_rn(dX, dX)));
                const bool na = ta && r2.x < pp.rc2f && r2.x >= pp.min_d2f;
                const bool nb = tb && r2.y < pp.rc2f && r2.y >= pp.min_d2f;
                const float2 ri = make_float2(rsqrtf(r2.x), rsqrtf(r2.y));
                const float2 re = __fadd2_rn(r2, EPS);
                const float2 rc = make_float2(__fdividef(1.f, re.x), __fdividef(1.f, re.y));
                // 1 / ((r^2 + eps^2) r) - L(r) / r^3
                float2 gsr;
                if (POLY) {
                    const float2 u = __ffma2_rn(r2, US, m1);
                    float2 nP = make_float2(pp.pc[kPPPoly], pp.pc[kPPPoly]);
#pragma unroll
                    for (int c = kPPPoly - 1; c >= 0; --c) nP = __ffma2_rn(nP, u, make_float2(pp.pc[c], pp.pc[c]));
                    gsr = __ffma2_rn(ri, rc, nP);
                } else {
                    const float2 uu = __fmul2_rn(__fmul2_rn(r2, ri), INV);
                    const int ka = max(min(static_cast<int>(uu.x), kPPTable - 1), 0);
                    const int kb = max(min(static_cast<int>(uu.y), kPPTable - 1), 0);
                    const float2 fr = __ffma2_rn(make_float2(static_cast<float>(ka), static_cast<float>(kb)), m1, uu);
                    const float2 t0 = make_float2(tabf[ka], tabf[kb]), t1 = make_float2(tabf[ka + 1], tabf[kb + 1]);
                    const float2 L = __ffma2_rn(fr, __ffma2_rn(t0, m1, t1), t0);
                    const float2 nri2 = __fmul2_rn(ri, __fmul2_rn(ri, m1));           // -1 / r^2
                    gsr = __fmul2_rn(__ffma2_rn(L, nri2, rc), ri);
                }
                // kc q_j times that (zq.zw = kc q)
                const float2 f = __fmul2_rn(gsr, make_float2(zq.z, zq.w));
                const float2 sc = make_float2(na ? f.x : 0.f, nb ? f.y : 0.f);
                E2x = __ffma2_rn(dX, sc, E2x);
                E2y = __ffma2_rn(dY, sc, E2y);
                E2z = __ffma2_rn(dZ, sc, E2z);
            };
            // slot range [sa, sb) of column (cx, cy) for this ion (dxa: its
            // distance to the column's x slab)
            auto column = [&](int cx, float dxa, int cy, uint32_t& sa, uint32_t& sb) {
                sa = 0u;
                sb = 0u;
                const float dya = fmaxf(0.f, fmaxf(static_cast<float>(cy) * h1 - fyi,
                                                   fyi - static_cast<float>(cy + 1) * h1));
                const float rem = rcpad - dxa * dxa - dya * dya;
                if (rem > 0.f) {
                    const float dzm = sqrtf(rem) + zpad;
                    const int za = max(z0, static_cast<int>(floorf((fzi - dzm) * ih2)));
                    const int zb = min(z1, static_cast<int>(floorf((fzi + dzm) * ih2)));
                    if (za <= zb) {
                        const uint32_t row = (static_cast<uint32_t>(cx) * g.n1 + static_cast<uint32_t>(cy)) * g.n2;
                        sa = start[row + static_cast<uint32_t>(za)];
                        sb = start[row + static_cast<uint32_t>(zb) + 1u];
                    }
                }
            };
            auto slab = [&](int cx) {
                return fmaxf(0.f, fmaxf(static_cast<float>(cx) * h0 - fxi, fxi - static_cast<float>(cx + 1) * h0));
            };
            const int wx0 = __reduce_min_sync(full, act ? x0 : INT_MAX);
            const int wx1 = __reduce_max_sync(full, act ? x1 : INT_MIN);
            const int wy0 = __reduce_min_sync(full, act ? y0 : INT_MAX);
            const int wy1 = __reduce_max_sync(full, act ? y1 : INT_MIN);
            for (int cx = wx0; cx <= wx1; ++cx) {
                const float dxa = slab(cx);
                for (int cy = wy0; cy <= wy1; ++cy) {
                    uint32_t sa = 0u, sb = 0u;
                    if (act && cx >= x0 && cx <= x1 && cy >= y0 && cy <= y1) column(cx, dxa, cy, sa, sb);
                    const bool has = sb > sa;
                    const uint32_t usa = __reduce_min_sync(full, has ? sa : 0xffffffffu);
                    const uint32_t usb = __reduce_max_sync(full, has ? sb : 0u);
                    if (usb <= usa) continue;                  // no lane has pairs in this column
                    const uint32_t len = __reduce_max_sync(full, sb - sa);
                    if (usb - usa <= len + (len >> 3) + 2u) {
                        for (uint32_t k = usa >> 1; 2u * k < usb; ++k)
                            pair2(k, 2u * k >= sa && 2u * k < sb, 2u * k + 1u >= sa && 2u * k + 1u < sb);
                    } else {
                        for (uint32_t k = sa >> 1; 2u * k < sb; ++k) pair2(k, 2u * k >= sa, 2u * k + 1u < sb);
                    }
                }
            }
            const float Ef[3] = {E2x.x + E2x.y, E2y.x + E2y.y, E2z.x + E2z.y};
#pragma unroll
            for (int c = 0; c < 3; ++c) E[c] += static_cast<double>(Ef[c]);
        } else if (!POLY) {
        const float4 own = pf[s];
        for (int cx = x0; cx <= x1; ++cx) {
            for (int cy = y0; cy <= y1; ++cy) {
                const uint32_t row = (static_cast<uint32_t>(cx) * g.n1 + static_cast<uint32_t>(cy)) * g.n2;
                const uint32_t sa = start[row + static_cast<uint32_t>(z0)];
                const uint32_t sb = start[row + static_cast<uint32_t>(z1) + 1u];
                for (uint32_t s2 = sa; s2 < sb; ++s2) {
                    const float4 qf = pf[s2];
                    const float ex0 = own.x - qf.x, ey0 = own.y - qf.y, ez0 = own.z - qf.z;
                    if (ex0 * ex0 + ey0 * ey0 + ez0 * ez0 >= pp.rc2_pre) continue;
                    const double4 pj = ps[s2];
                    const double dx = xi - pj.x, dy = yi - pj.y, dz = zi - pj.z;
                    const double r2 = dx * dx + dy * dy + dz * dz;
                    if (s2 == s || r2 < pp.min_d2 || r2 >= pp.rc2) continue;
                    const double r = sqrt(r2);
                    const double u = r * pp.inv_dr;
                    const int kt = min(static_cast<int>(u), kPPTable - 1);
                    const double fr = u - kt;
                    const double L = fma(fr, tab[kt + 1] - tab[kt], tab[kt]);
                    // softened direct field minus the mesh's long-range part, / r
                    const double sc = kCoulomb * (1.0 / (r2 + pp.eps2) - L / r2) / r * pj.w;
                    E[0] += dx * sc;
                    E[1] += dy * sc;
                    E[2] += dz * sc;
                }
            }
        }
        }
    }
    if (!act) {
        if (in_range) { ex[i] = 0.0; ey[i] = 0.0; ez[i] = 0.0; }
        return;
    }
    ex[i] = E[0]; ey[i] = E[1]; ez[i] = E[2];
}

// Field of every ion, one thread per ion in sorted order (blocks of
// consecutive ions share their partners in L1).  The polynomial form runs
// blocks of 128: finer blocks leave fewer warps waiting for their block's
// slowest one (the cloud's dense middle costs many times its edges).
template <bool REF_WEIGHTS, class GT, bool POLY = false>
__global__ void __launch_bounds__(POLY ? 128 : 256, POLY ? 8 : 4) k_sc_gather(MeshGeom g, PPParams pp,
                            const double4* __restrict__ ps, const float4* __restrict__ pf,
                            const uint32_t* __restrict__ keys, const uint32_t* __restrict__ vals,
                            const uint32_t* __restrict__ start, uint32_t n, const uint32_t* __restrict__ slots,
                            const GT* __restrict__ gx, const GT* __restrict__ gy, const GT* __restrict__ gz,
                            double* __restrict__ ex, double* __restrict__ ey, double* __restrict__ ez) {
    // the long-range table (the polynomial form has none; it runs with the
    // float loop only)
    __shared__ double tab[(REF_WEIGHTS || POLY) ? 1 : kPPTable + 1];
    float* tabf = reinterpret_cast<float*>(tab);
    if (!REF_WEIGHTS && !POLY && pp.on) {
        if (pp.use_float) {
            for (int k = threadIdx.x; k <= kPPTable; k += blockDim.x) tabf[k] = static_cast<float>(pp.table[k]);
        } else {
            for (int k = threadIdx.x; k <= kPPTable; k += blockDim.x) tab[k] = pp.table[k];
        }
        __syncthreads();
    }
    sc_gather_ion<REF_WEIGHTS, GT, POLY>(blockIdx.x * blockDim.x + threadIdx.x, g, pp, ps, pf, keys, vals, start, n,
                                         slots, gx, gy, gz, ex, ey, ez, tab, tabf);
}

// L(r) / (a r)^3 as a function of x = (a r)^2: (erf(t) - 2t e^(-x) / sqrt(pi)) / t^3
// with t = sqrt(x); by its series (2/sqrt(pi)) sum_{n>=1} (-1)^(n+1)
// x^(n-1) 2n / (n! (2n+1)) below x = 1/4, where the difference cancels.
double long_range_ratio(double x) {
    if (x < 0.25) {
        double sum = 0.0, term = 1.0;                 // term = x^(n-1) / n!
        for (int n = 1; n < 24; ++n) {
            if (n > 1) term *= x / n;
            sum += ((n & 1) ? 1.0 : -1.0) * term * 2.0 * n / (2.0 * n + 1.0);
        }
        return 2.0 / std::sqrt(kPi) * sum;
    }
    const double t = std::sqrt(x);
    return (std::erf(t) - 2.0 * t / std::sqrt(kPi) * std::exp(-x)) / (x * t);
}

// The float loop's long-range term -L(r)/r^3 as a degree-kPPPoly polynomial
// in u = 2 r^2 / r_c^2 - 1: Chebyshev interpolation at kPPPoly + 1 nodes,
// rewritten in powers of u and rounded to float.  Accepted (pp.poly = 1)
// when, evaluated in float by Horner's rule as the kernel does, it is within
// 1e-5 of the short-range term 1/r^3 - L(r)/r^3 at every r of 4096 points
// in (0, r_c] (the table form's float rounding is ~2e-6 there); else the
// loop keeps the table.
void fit_long_range_poly(double alpha, double rc, PPParams& pp) {
    constexpr int N = kPPPoly + 1;
    const double X = alpha * alpha * rc * rc, a3 = alpha * alpha * alpha;
    double cheb[N];
    for (int k = 0; k < N; ++k) {
        double acc = 0.0;
        for (int j = 0; j < N; ++j) {
            const double th = kPi * (j + 0.5) / N;
            acc += a3 * long_range_ratio(0.5 * X * (std::cos(th) + 1.0)) * std::cos(k * th);
        }
        cheb[k] = (k == 0 ? 1.0 : 2.0) * acc / N;
    }
    // T_k in powers of u: T_0 = 1, T_1 = u, T_{k+1} = 2u T_k - T_{k-1}
    double mono[N] = {}, tm[N] = {}, t0[N] = {}, t1[N] = {};
    t0[0] = 1.0;
    t1[1] = 1.0;
    mono[0] = cheb[0];
    mono[1] = cheb[1];
    for (int k = 2; k < N; ++k) {
        for (int e = 0; e < N; ++e) tm[e] = (e > 0 ? 2.0 * t1[e - 1] : 0.0) - t0[e];
        for (int e = 0; e < N; ++e) { mono[e] += cheb[k] * tm[e]; t0[e] = t1[e]; t1[e] = tm[e]; }
    }
    for (int e = 0; e < N; ++e) pp.pc[e] = static_cast<float>(-mono[e]);
    pp.pu_s = static_cast<float>(2.0 / (rc * rc));
    double worst = 0.0;
    for (int i = 1; i <= 4096; ++i) {
        const double r = rc * i / 4096.0;
        const float u = std::fmaf(static_cast<float>(r * r), pp.pu_s, -1.0f);
        float np = pp.pc[kPPPoly];
        for (int e = kPPPoly - 1; e >= 0; --e) np = std::fmaf(np, u, pp.pc[e]);
        const double lr = a3 * long_range_ratio(alpha * alpha * r * r);
        worst = std::max(worst, std::fabs(-static_cast<double>(np) - lr) / std::fabs(1.0 / (r * r * r) - lr));
    }
    pp.poly = worst <= 1e-5 ? 1 : 0;
}

template <class T>
cudaError_t dev_alloc(T** p, size_t count) {
    *p = nullptr;
    if (count == 0) return cudaSuccess;
    return cudaMalloc(reinterpret_cast<void**>(p), count * sizeof(T));
}

inline unsigned blocks_for(size_t n, int threads) { return static_cast<unsigned>((n + threads - 1) / threads); }

}  // namespace

struct SpaceChargeSolver {
    int mode = ICB_SC_OFF;
    MeshGeom g{};
    double h[3] = {0, 0, 0};
    PPParams pp{};
    uint32_t cap = 0;
    int key_bits = 1;
    uint32_t* keys = nullptr;
    uint32_t* keys_sorted = nullptr;
    uint32_t* vals = nullptr;
    uint32_t* vals_sorted = nullptr;
    uint32_t* start = nullptr;
    double4* ps = nullptr;
    float4* pf = nullptr;
    double* pp_table = nullptr;
    void* cub_tmp = nullptr;
    size_t cub_bytes = 0;
    double* rho = nullptr;
    cufftDoubleComplex* rho_hat = nullptr;
    cufftDoubleComplex* tmp_hat = nullptr;
    double* egrid[3] = {nullptr, nullptr, nullptr};
    cufftDoubleComplex* ghat[3] = {nullptr, nullptr, nullptr};
    double* esc[3] = {nullptr, nullptr, nullptr};
    cufftHandle fwd = 0, inv = 0, inv3 = 0;
    bool have_fwd = false, have_inv = false, have_inv3 = false;
    // single-precision mesh (isolated solver in the float forms): the
    // charge and the field grids hold the planes x < n0 only (the mesh);
    // the transform runs as a 2D (y, z) pass over those planes and a 1D x
    // pass over the whole spectrum, forward and inverse
    bool f32 = false;
    float* rho_f = nullptr;               // n0 x m1 x m2, zero outside the mesh
    cufftComplex* rho_hat_f = nullptr;
    cufftComplex* tmp_hat_f = nullptr;
    float* egrid_f = nullptr;             // three grids of n0 x m1 x m2, one block
    float* gfold_f = nullptr;             // three folded kernels, one block
    cufftHandle xpass = 0, inv2 = 0;
    bool have_xpass = false, have_inv2 = false;
    // a padded x length of 256 runs the fused x pass (k_sc_xconv) in place
    // of the cuFFT x passes and the separate kernel products
    bool xfused = false;
    float2* tw256 = nullptr;
    // other devices' ions in this solve (icb_spacecharge_set_peers); cap
    // covers own_cap own ions plus the peers
    uint32_t own_cap = 0;
    PeerIons peers{};
    uint32_t* own_flag = nullptr;          // per sorted slot, then its scan
    uint32_t* own_pos = nullptr;
    uint32_t* own_slots = nullptr;         // sorted slots of the own ions
    void* scan_tmp = nullptr;
    size_t scan_bytes = 0;

    ~SpaceChargeSolver() {
        for (void* p : {static_cast<void*>(own_flag), static_cast<void*>(own_pos), static_cast<void*>(own_slots),
                        scan_tmp})
            if (p) cudaFree(p);
        if (have_fwd) cufftDestroy(fwd);
        if (have_inv) cufftDestroy(inv);
        if (have_inv3) cufftDestroy(inv3);
        if (have_xpass) cufftDestroy(xpass);
        if (have_inv2) cufftDestroy(inv2);
        for (void* p : {static_cast<void*>(keys), static_cast<void*>(keys_sorted), static_cast<void*>(vals),
                        static_cast<void*>(vals_sorted), static_cast<void*>(start), static_cast<void*>(ps), static_cast<void*>(pf), static_cast<void*>(pp_table),
                        cub_tmp,
                        static_cast<void*>(rho), static_cast<void*>(rho_hat), static_cast<void*>(tmp_hat)})
            if (p) cudaFree(p);
        if (egrid[0]) cudaFree(egrid[0]);   // one block holds the three grids
        for (void* q : {static_cast<void*>(rho_f), static_cast<void*>(rho_hat_f), static_cast<void*>(tmp_hat_f),
                        static_cast<void*>(egrid_f), static_cast<void*>(gfold_f), static_cast<void*>(tw256)})
            if (q) cudaFree(q);
        for (int c = 0; c < 3; ++c) {
            if (ghat[c]) cudaFree(ghat[c]);
            if (esc[c]) cudaFree(esc[c]);
        }
    }
    size_t real_size() const { return static_cast<size_t>(g.m0) * g.m1 * g.m2; }
    size_t mesh_planes_size() const { return static_cast<size_t>(g.n0) * g.m1 * g.m2; }
    size_t cplx_size() const { return static_cast<size_t>(g.m0) * g.m1 * (g.m2 / 2 + 1); }
};

#define SC_CUDA(expr)                                                                          \
    do {                                                                                       \
        cudaError_t e_ = (expr);                                                               \
        if (e_ != cudaSuccess) {                                                               \
            err = std::string(#expr) + ": " + cudaGetErrorString(e_);                          \
            return e_ == cudaErrorMemoryAllocation ? ICB_ERR_OUT_OF_MEMORY : ICB_ERR_CUDA;     \
        }                                                                                      \
    } while (0)
#define SC_FFT(expr)                                                                           \
    do {                                                                                       \
        cufftResult r_ = (expr);                                                               \
        if (r_ != CUFFT_SUCCESS) {                                                             \
            err = std::string(#expr) + ": cuFFT error " + std::to_string(static_cast<int>(r_)); \
            return r_ == CUFFT_ALLOC_FAILED ? ICB_ERR_OUT_OF_MEMORY : ICB_ERR_CUDA;            \
        }                                                                                      \
    } while (0)

int sc_create(const icb_spacecharge_config& c, uint64_t n_ions, bool pp_float, cudaStream_t s,
              SpaceChargeSolver** out, std::string& err) {
    *out = nullptr;
    if (c.mode != ICB_SC_P3M_ISOLATED && c.mode != ICB_SC_PM_PERIODIC_REF) {
        err = "unknown space-charge mode";
        return ICB_ERR_INVALID_ARGUMENT;
    }
    const bool iso = c.mode == ICB_SC_P3M_ISOLATED;
    const int nmax = iso ? 256 : 512;
    for (int a = 0; a < 3; ++a) {
        if (c.grid_n[a] < 8 || c.grid_n[a] > nmax) {
            err = "grid_n must be in [8, " + std::to_string(nmax) + "] per axis";
            return ICB_ERR_INVALID_ARGUMENT;
        }
        if (!(c.box_max_m[a] > c.box_min_m[a])) {
            err = "box_max_m must exceed box_min_m on every axis";
            return ICB_ERR_INVALID_ARGUMENT;
        }
    }
    if (n_ions == 0 || n_ions >= (1ull << 31)) {
        err = "space charge needs 1 .. 2^31-1 ions";
        return ICB_ERR_INVALID_ARGUMENT;
    }
    auto sv = std::make_unique<SpaceChargeSolver>();
    SpaceChargeSolver& S = *sv;
    S.mode = c.mode;
    MeshGeom& g = S.g;
    g.n0 = c.grid_n[0]; g.n1 = c.grid_n[1]; g.n2 = c.grid_n[2];
    g.m0 = iso ? 2 * g.n0 : g.n0; g.m1 = iso ? 2 * g.n1 : g.n1; g.m2 = iso ? 2 * g.n2 : g.n2;
    g.lo0 = c.box_min_m[0]; g.lo1 = c.box_min_m[1]; g.lo2 = c.box_min_m[2];
    double hmax = 0.0;
    for (int a = 0; a < 3; ++a) {
        const double ext = c.box_max_m[a] - c.box_min_m[a];
        S.h[a] = ext / c.grid_n[a];
        hmax = std::max(hmax, S.h[a]);
    }
    if (iso) {
        g.ih0 = 1.0 / S.h[0]; g.ih1 = 1.0 / S.h[1]; g.ih2 = 1.0 / S.h[2];
    } else {
        // GPUSpaceChargeP3M.cu: inv_spacing = grid_n / domain_size
        g.ih0 = c.grid_n[0] / (c.box_max_m[0] - c.box_min_m[0]);
        g.ih1 = c.grid_n[1] / (c.box_max_m[1] - c.box_min_m[1]);
        g.ih2 = c.grid_n[2] / (c.box_max_m[2] - c.box_min_m[2]);
    }
    g.ncell = static_cast<uint32_t>(g.n0) * g.n1 * g.n2;
    S.key_bits = 1;
    while ((1ull << S.key_bits) <= g.ncell) ++S.key_bits;
    S.pp.on = iso ? 1 : 0;
    if (iso) {
        const double ah = c.alpha_h > 0.0 ? c.alpha_h : 1.0;
        const double rcc = c.pp_cutoff_cells > 0.0 ? c.pp_cutoff_cells : 2.0;
        const double soft = c.softening_m < 0.0 ? 1e-10 : c.softening_m;
        S.pp.alpha = ah / hmax;
        const double rc = rcc * hmax;
        S.pp.rc2 = rc * rc;
        S.pp.r0 = static_cast<int>(std::ceil(rc / S.h[0]));
        S.pp.r1 = static_cast<int>(std::ceil(rc / S.h[1]));
        S.pp.r2 = static_cast<int>(std::ceil(rc / S.h[2]));
        S.pp.eps2 = soft * soft;
        S.pp.min_d2 = std::max(soft * soft * 1e-4, 1e-30);
        S.pp.inv_dr = kPPTable / rc;
        S.pp.use_float = pp_float ? 1 : 0;
        S.pp.rc2f = static_cast<float>(rc * rc);
        S.pp.eps2f = static_cast<float>(S.pp.eps2);
        S.pp.min_d2f = static_cast<float>(S.pp.min_d2);
        S.pp.inv_drf = static_cast<float>(S.pp.inv_dr);
        // float positions relative to the mesh origin carry an absolute error
        // below 1e-7 of the box; the margin keeps every pair under r_c
        S.pp.rc2_pre = static_cast<float>(rc * rc * 1.001 + 1e-6 * 3.0 * (c.box_max_m[0] - c.box_min_m[0]) * rc);
        if (pp_float) fit_long_range_poly(S.pp.alpha, rc, S.pp);
    }
    S.cap = static_cast<uint32_t>(n_ions);
    S.own_cap = S.cap;
    SC_CUDA(dev_alloc(&S.keys, S.cap));
    SC_CUDA(dev_alloc(&S.keys_sorted, S.cap));
    SC_CUDA(dev_alloc(&S.vals, S.cap));
    SC_CUDA(dev_alloc(&S.vals_sorted, S.cap));
    SC_CUDA(dev_alloc(&S.start, static_cast<size_t>(g.ncell) + 1));
    SC_CUDA(dev_alloc(&S.ps, S.cap));
    SC_CUDA(dev_alloc(&S.pf, static_cast<size_t>(S.cap) + 1));
    SC_CUDA(cudaMemsetAsync(S.pf, 0, (static_cast<size_t>(S.cap) + 1) * sizeof(float4), s));
    if (iso) {
        std::vector<double> tab(kPPTable + 1);
        const double a = S.pp.alpha;
        for (int k = 0; k <= kPPTable; ++k) {
            const double r = k / S.pp.inv_dr;
            tab[k] = std::erf(a * r) - (2.0 * a * r / std::sqrt(kPi)) * std::exp(-a * a * r * r);
        }
        SC_CUDA(dev_alloc(&S.pp_table, tab.size()));
        SC_CUDA(cudaMemcpy(S.pp_table, tab.data(), tab.size() * sizeof(double), cudaMemcpyHostToDevice));
        S.pp.table = S.pp_table;
    }
    SC_CUDA(cub::DeviceRadixSort::SortPairs(nullptr, S.cub_bytes, S.keys, S.keys_sorted, S.vals, S.vals_sorted,
                                            static_cast<int>(S.cap), 0, S.key_bits, s));
    SC_CUDA(cudaMalloc(&S.cub_tmp, std::max<size_t>(S.cub_bytes, 16)));
    const bool f32 = iso && pp_float;
    S.f32 = f32;
    for (int a = 0; a < 3; ++a) SC_CUDA(dev_alloc(&S.esc[a], S.cap));
    // the double grid and forward plan serve the transformed field kernels
    // (always built in FP64) and the FP64 per-step path
    SC_CUDA(dev_alloc(&S.rho, S.real_size()));
    SC_FFT(cufftPlan3d(&S.fwd, g.m0, g.m1, g.m2, CUFFT_D2Z));
    S.have_fwd = true;
    SC_FFT(cufftSetStream(S.fwd, s));
    if (!f32) {
        SC_CUDA(dev_alloc(&S.rho_hat, S.cplx_size()));
        SC_CUDA(dev_alloc(&S.egrid[0], 3 * S.real_size()));
        for (int a = 0; a < 3; ++a) S.egrid[a] = S.egrid[0] + a * S.real_size();
        SC_FFT(cufftPlan3d(&S.inv, g.m0, g.m1, g.m2, CUFFT_Z2D));
        S.have_inv = true;
        SC_FFT(cufftSetStream(S.inv, s));
    }
    if (iso) {
        int dims[3] = {g.m0, g.m1, g.m2};
        cufftDoubleComplex* tmp = nullptr;
        if (!f32) {
            // the three field components go through one batched inverse transform
            SC_FFT(cufftPlanMany(&S.inv3, 3, dims, nullptr, 1, 0, nullptr, 1, 0, CUFFT_Z2D, 3));
            S.have_inv3 = true;
            SC_FFT(cufftSetStream(S.inv3, s));
            SC_CUDA(dev_alloc(&S.tmp_hat, 3 * S.cplx_size()));
        } else {
            SC_CUDA(dev_alloc(&tmp, S.cplx_size()));
            SC_CUDA(dev_alloc(&S.gfold_f, 3 * fold_geom(g).n));
        }
        for (int a = 0; a < 3; ++a) {
            cufftDoubleComplex* gh = tmp;
            if (!f32) {
                SC_CUDA(dev_alloc(&S.ghat[a], S.cplx_size()));
                gh = S.ghat[a];
            }
            k_sc_green<<<blocks_for(S.real_size(), 256), 256, 0, s>>>(g, S.h[0], S.h[1], S.h[2], S.pp.alpha, a, S.rho);
            SC_CUDA(cudaGetLastError());
            SC_FFT(cufftExecD2Z(S.fwd, S.rho, gh));
            k_sc_normalize<<<blocks_for(S.cplx_size(), 256), 256, 0, s>>>(g, gh);
            SC_CUDA(cudaGetLastError());
            if (f32) {
                const size_t nf = fold_geom(g).n;
                k_sc_fold<<<blocks_for(nf, 256), 256, 0, s>>>(g, gh, g.m0 == kXLen ? 1 : 0, S.gfold_f + a * nf);
                SC_CUDA(cudaGetLastError());
            }
        }
        if (f32) {
            // single-precision per-step mesh.  Forward: 2D R2C over (y, z)
            // of the n0 mesh planes, then the x pass over every (y, kz)
            // column (the planes x >= n0 are zero).  Inverse per component:
            // the x pass, then the 2D C2R of the planes x < n0 only (the
            // gather reads nothing else).
            SC_CUDA(cudaStreamSynchronize(s));
            cudaFree(tmp);
            cudaFree(S.rho);
            S.rho = nullptr;
            cufftDestroy(S.fwd);
            S.have_fwd = false;
            SC_CUDA(dev_alloc(&S.rho_f, S.mesh_planes_size()));
            SC_CUDA(dev_alloc(&S.rho_hat_f, S.cplx_size()));
            SC_CUDA(dev_alloc(&S.tmp_hat_f, 3 * S.cplx_size()));
            SC_CUDA(dev_alloc(&S.egrid_f, 3 * S.mesh_planes_size()));
            // the deposit writes every mesh node; the rest stays zero (an
            // out-of-place R2C leaves its input as it is)
            SC_CUDA(cudaMemsetAsync(S.rho_f, 0, S.mesh_planes_size() * sizeof(float), s));
            int n2d[2] = {g.m1, g.m2};
            SC_FFT(cufftPlanMany(&S.fwd, 2, n2d, nullptr, 1, 0, nullptr, 1, 0, CUFFT_R2C, g.n0));
            S.have_fwd = true;
            SC_FFT(cufftSetStream(S.fwd, s));
            S.xfused = g.m0 == kXLen;
            if (S.xfused) {
                std::vector<float2> tw(kXLen);
                for (int m = 0; m < kXLen; ++m)
                    tw[m] = make_float2(static_cast<float>(std::cos(2.0 * kPi * m / kXLen)),
                                        static_cast<float>(-std::sin(2.0 * kPi * m / kXLen)));
                SC_CUDA(dev_alloc(&S.tw256, kXLen));
                SC_CUDA(cudaMemcpy(S.tw256, tw.data(), kXLen * sizeof(float2), cudaMemcpyHostToDevice));
            } else {
                int n1d[1] = {g.m0};
                const int cols = g.m1 * (g.m2 / 2 + 1);
                SC_FFT(cufftPlanMany(&S.xpass, 1, n1d, n1d, cols, 1, n1d, cols, 1, CUFFT_C2C, cols));
                S.have_xpass = true;
                SC_FFT(cufftSetStream(S.xpass, s));
            }
            // the fused x pass leaves the three components' mesh planes
            // back to back: one inverse over all of them
            SC_FFT(cufftPlanMany(&S.inv2, 2, n2d, nullptr, 1, 0, nullptr, 1, 0, CUFFT_C2R,
                                 S.xfused ? 3 * g.n0 : g.n0));
            S.have_inv2 = true;
            SC_FFT(cufftSetStream(S.inv2, s));
        }
    }
    SC_CUDA(cudaStreamSynchronize(s));
    *out = sv.release();
    return ICB_OK;
}

void sc_destroy(SpaceChargeSolver* S) { delete S; }

int sc_set_peers(SpaceChargeSolver* S, const double* xyzq, uint64_t n, uint64_t skip_b, uint64_t skip_n,
                 cudaStream_t s, std::string& err) {
    if (n == 0) {
        S->peers = PeerIons{};
        return ICB_OK;
    }
    if (S->mode != ICB_SC_P3M_ISOLATED) {
        err = "peer ions need the isolated P3M solver";
        return ICB_ERR_UNSUPPORTED;
    }
    if (xyzq == nullptr || (reinterpret_cast<uintptr_t>(xyzq) & 15u) != 0u) {
        err = "peer ions: null or misaligned device array (16-byte aligned x, y, z, q quadruples)";
        return ICB_ERR_INVALID_ARGUMENT;
    }
    if (skip_b > n || skip_n > n - skip_b || static_cast<uint64_t>(S->own_cap) + n >= (1ull << 31)) {
        err = "peer ions: skip range outside the list, or more than 2^31 ions in the solve";
        return ICB_ERR_INVALID_ARGUMENT;
    }
    const uint64_t total = static_cast<uint64_t>(S->own_cap) + n;
    if (total > S->cap || S->own_slots == nullptr) {
        // grow the sort, permutation and slot buffers to own + peers
        SC_CUDA(cudaStreamSynchronize(s));
        const uint32_t cap = static_cast<uint32_t>(std::max<uint64_t>(total, S->cap));
        for (void** p : {reinterpret_cast<void**>(&S->keys), reinterpret_cast<void**>(&S->keys_sorted),
                         reinterpret_cast<void**>(&S->vals), reinterpret_cast<void**>(&S->vals_sorted),
                         reinterpret_cast<void**>(&S->ps), reinterpret_cast<void**>(&S->pf), &S->cub_tmp,
                         reinterpret_cast<void**>(&S->own_flag), reinterpret_cast<void**>(&S->own_pos),
                         reinterpret_cast<void**>(&S->own_slots), &S->scan_tmp}) {
            if (*p) cudaFree(*p);
            *p = nullptr;
        }
        S->cap = cap;
        SC_CUDA(dev_alloc(&S->keys, cap));
        SC_CUDA(dev_alloc(&S->keys_sorted, cap));
        SC_CUDA(dev_alloc(&S->vals, cap));
        SC_CUDA(dev_alloc(&S->vals_sorted, cap));
        SC_CUDA(dev_alloc(&S->ps, cap));
        SC_CUDA(dev_alloc(&S->pf, static_cast<size_t>(cap) + 1));
        SC_CUDA(cudaMemsetAsync(S->pf, 0, (static_cast<size_t>(cap) + 1) * sizeof(float4), s));
        SC_CUDA(dev_alloc(&S->own_flag, cap));
        SC_CUDA(dev_alloc(&S->own_pos, cap));
        SC_CUDA(dev_alloc(&S->own_slots, S->own_cap));
        S->cub_bytes = 0;
        SC_CUDA(cub::DeviceRadixSort::SortPairs(nullptr, S->cub_bytes, S->keys, S->keys_sorted, S->vals,
                                                S->vals_sorted, static_cast<int>(cap), 0, S->key_bits, s));
        SC_CUDA(cudaMalloc(&S->cub_tmp, std::max<size_t>(S->cub_bytes, 16)));
        S->scan_bytes = 0;
        SC_CUDA(cub::DeviceScan::ExclusiveSum(nullptr, S->scan_bytes, S->own_flag, S->own_pos, static_cast<int>(cap), s));
        SC_CUDA(cudaMalloc(&S->scan_tmp, std::max<size_t>(S->scan_bytes, 16)));
    }
    S->peers.xyzq = reinterpret_cast<const double4*>(xyzq);
    S->peers.n = static_cast<uint32_t>(n);
    S->peers.skip_b = static_cast<uint32_t>(skip_b);
    S->peers.skip_n = static_cast<uint32_t>(skip_n);
    return ICB_OK;
}

int sc_export(const double* x, const double* y, const double* z, const double* q, const uint8_t* flags, uint64_t n,
              double* out, cudaStream_t s, std::string& err) {
    if (out == nullptr || (reinterpret_cast<uintptr_t>(out) & 15u) != 0u) {
        err = "export: null or misaligned device array (16-byte aligned x, y, z, q quadruples)";
        return ICB_ERR_INVALID_ARGUMENT;
    }
    k_sc_export<<<blocks_for(n, 256), 256, 0, s>>>(x, y, z, q, flags, n, reinterpret_cast<double4*>(out));
    SC_CUDA(cudaGetLastError());
    return ICB_OK;
}

int sc_solve(SpaceChargeSolver* S, const double* x, const double* y, const double* z, const double* q,
             const uint8_t* flags, uint64_t n, cudaStream_t s, std::string& err) {
    if (n > S->own_cap) {
        err = "more ions than the space-charge solver was configured for";
        return ICB_ERR_STATE;
    }
    const MeshGeom& g = S->g;
    const bool iso = S->mode == ICB_SC_P3M_ISOLATED;
    const uint32_t n_own = static_cast<uint32_t>(n);
    const uint32_t nn = n_own + S->peers.n;     // sorted slots: own ions and peers
    SC_FFT(cufftSetStream(S->fwd, s));
    if (S->have_inv) SC_FFT(cufftSetStream(S->inv, s));
    if (S->have_inv3) SC_FFT(cufftSetStream(S->inv3, s));
    if (S->have_xpass) SC_FFT(cufftSetStream(S->xpass, s));
    if (S->have_inv2) SC_FFT(cufftSetStream(S->inv2, s));
    k_sc_bin<<<blocks_for(nn, 256), 256, 0, s>>>(g, x, y, z, flags, n_own, S->peers, iso ? 0 : 1, S->keys, S->vals);
    SC_CUDA(cudaGetLastError());
    size_t bytes = S->cub_bytes;
    SC_CUDA(cub::DeviceRadixSort::SortPairs(S->cub_tmp, bytes, S->keys, S->keys_sorted, S->vals, S->vals_sorted,
                                            static_cast<int>(nn), 0, S->key_bits, s));
    k_sc_cell_start<<<blocks_for((static_cast<size_t>(g.ncell) + 4) / 4, 256), 256, 0, s>>>(S->keys_sorted, nn,
                                                                                            g.ncell, S->start);
    SC_CUDA(cudaGetLastError());
    k_sc_permute<<<blocks_for(nn, 256), 256, 0, s>>>(g, x, y, z, q, S->vals_sorted, nn, n_own, S->peers,
                                                     (S->pp.on && S->pp.use_float) ? 1 : 0, S->ps, S->pf);
    SC_CUDA(cudaGetLastError());
    // with peers the gather runs over this handle's ions only, in sorted order
    const uint32_t* slots = nullptr;
    uint32_t n_gather = nn;
    if (S->peers.n > 0) {
        k_sc_own_flag<<<blocks_for(nn, 256), 256, 0, s>>>(S->vals_sorted, nn, n_own, S->own_flag);
        SC_CUDA(cudaGetLastError());
        size_t sb = S->scan_bytes;
        SC_CUDA(cub::DeviceScan::ExclusiveSum(S->scan_tmp, sb, S->own_flag, S->own_pos, static_cast<int>(nn), s));
        k_sc_own_scatter<<<blocks_for(nn, 256), 256, 0, s>>>(S->vals_sorted, S->own_pos, nn, n_own, S->own_slots);
        SC_CUDA(cudaGetLastError());
        slots = S->own_slots;
        n_gather = n_own;
    }
    const size_t mesh_nodes = static_cast<size_t>(g.n0) * g.n1 * g.n2;
    if (iso && S->f32) {
        const size_t cs = S->cplx_size(), ms = S->mesh_planes_size();
        const size_t upper = cs / 2;           // planes x >= n0 of the (y, kz) spectrum
        k_sc_deposit<false, float><<<blocks_for(mesh_nodes, 256), 256, 0, s>>>(g, S->ps, S->start, S->rho_f);
        SC_CUDA(cudaGetLastError());
        SC_FFT(cufftExecR2C(S->fwd, S->rho_f, S->rho_hat_f));
        if (S->xfused) {
            const size_t P = static_cast<size_t>(g.m1) * (g.m2 / 2 + 1);
            k_sc_xconv<<<blocks_for(P, kXCols), 256, 0, s>>>(g, S->rho_hat_f, S->gfold_f, S->tw256, S->tmp_hat_f);
            SC_CUDA(cudaGetLastError());
            SC_FFT(cufftExecC2R(S->inv2, S->tmp_hat_f, S->egrid_f));
        } else {
        SC_CUDA(cudaMemsetAsync(S->rho_hat_f + upper, 0, (cs - upper) * sizeof(cufftComplex), s));
        SC_FFT(cufftExecC2C(S->xpass, S->rho_hat_f, S->rho_hat_f, CUFFT_FORWARD));
        const size_t nf = fold_geom(g).n;
        k_sc_cmul_fold<<<blocks_for(nf, 256), 256, 0, s>>>(g, S->rho_hat_f, S->gfold_f, S->tmp_hat_f);
        SC_CUDA(cudaGetLastError());
        for (int c = 0; c < 3; ++c) {
            SC_FFT(cufftExecC2C(S->xpass, S->tmp_hat_f + c * cs, S->tmp_hat_f + c * cs, CUFFT_INVERSE));
            SC_FFT(cufftExecC2R(S->inv2, S->tmp_hat_f + c * cs, S->egrid_f + c * ms));
        }
        }
        auto gather = S->pp.poly ? k_sc_gather<false, float, true> : k_sc_gather<false, float, false>;
        const int gb = S->pp.poly ? 128 : 256;
        gather<<<blocks_for(n_gather, gb), gb, 0, s>>>(
            g, S->pp, S->ps, S->pf, S->keys_sorted, S->vals_sorted, S->start, n_gather, slots, S->egrid_f,
            S->egrid_f + ms, S->egrid_f + 2 * ms, S->esc[0], S->esc[1], S->esc[2]);
        SC_CUDA(cudaGetLastError());
    } else if (iso) {
        SC_CUDA(cudaMemsetAsync(S->rho, 0, S->real_size() * sizeof(double), s));
        k_sc_deposit<false, double><<<blocks_for(mesh_nodes, 256), 256, 0, s>>>(g, S->ps, S->start, S->rho);
        SC_CUDA(cudaGetLastError());
        SC_FFT(cufftExecD2Z(S->fwd, S->rho, S->rho_hat));
        k_sc_cmul3<cufftDoubleComplex><<<blocks_for(S->cplx_size(), 256), 256, 0, s>>>(S->rho_hat, S->ghat[0], S->ghat[1], S->ghat[2],
                                                                    S->tmp_hat, S->cplx_size());
        SC_CUDA(cudaGetLastError());
        SC_FFT(cufftExecZ2D(S->inv3, S->tmp_hat, S->egrid[0]));
        k_sc_gather<false, double><<<blocks_for(n_gather, 256), 256, 0, s>>>(
            g, S->pp, S->ps, S->pf, S->keys_sorted, S->vals_sorted, S->start, n_gather, slots, S->egrid[0],
            S->egrid[1], S->egrid[2], S->esc[0], S->esc[1], S->esc[2]);
        SC_CUDA(cudaGetLastError());
    } else {
        k_sc_deposit<true, double><<<blocks_for(mesh_nodes, 256), 256, 0, s>>>(g, S->ps, S->start, S->rho);
        SC_CUDA(cudaGetLastError());
        SC_FFT(cufftExecD2Z(S->fwd, S->rho, S->rho_hat));
        k_sc_poisson_ref<<<blocks_for(S->cplx_size(), 256), 256, 0, s>>>(g, S->h[0], S->h[1], S->h[2], S->rho_hat);
        SC_CUDA(cudaGetLastError());
        // the potential lands in rho (no longer needed after the forward FFT)
        SC_FFT(cufftExecZ2D(S->inv, S->rho_hat, S->rho));
        const double scale = 1.0 / static_cast<double>(S->real_size());
        k_sc_efield_ref<<<blocks_for(S->real_size(), 256), 256, 0, s>>>(g, S->h[0], S->h[1], S->h[2], scale, S->rho,
                                                                         S->egrid[0], S->egrid[1], S->egrid[2]);
        SC_CUDA(cudaGetLastError());
        k_sc_gather<true, double><<<blocks_for(n_gather, 256), 256, 0, s>>>(
            g, S->pp, S->ps, S->pf, S->keys_sorted, S->vals_sorted, S->start, n_gather, slots, S->egrid[0],
            S->egrid[1], S->egrid[2], S->esc[0], S->esc[1], S->esc[2]);
        SC_CUDA(cudaGetLastError());
    }
    return ICB_OK;
}

const double* sc_field(const SpaceChargeSolver* S, int axis) { return S->esc[axis]; }

int sc_kernel_count(const SpaceChargeSolver* S) {
    // kernels of one solve that this library launches (cuFFT, CUB and
    // memsets not counted): bin, cell starts, permute, deposit, then the
    // kernel products (or the fused x pass) and the gather, or the
    // reference's Poisson step, its differences and the gather; with peer
    // ions also the own-slot flag and scatter
    const int peers = S->peers.n > 0 ? 2 : 0;
    return (S->mode == ICB_SC_P3M_ISOLATED ? 4 + 1 + 1 : 4 + 1 + 1 + 1) + peers;
}

}  // namespace icb
