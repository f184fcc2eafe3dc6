// Direct (all-pairs) sums: the pair loops of DirectSum::meshSolve (src/LpmDirectSum.cpp:94-167)
// and DirectSum::meshfreeSolve (src/LpmDirectSum.cpp:175-254) as shared-memory-tiled sm_100a
// kernels.
//
// Layout: sources are packed n x 4 (x, y, z, w) with w = strength (vorticity * area, or charge);
// a block stages SRC_TILE sources in shared memory and every thread sweeps them against its
// TPT register-resident targets, so each source is read once per block from HBM/L2 and once
// per thread from shared memory as a broadcast 128-bit load.
//
// FP64 kernels follow the reference formula term by term: den = (R^2 - x.y) + delta^2, the term
// is dropped when |den| <= 1e-13 (src/LpmVectorKernel.h:24-28).  The sum is reorganised as
// u = mult * (x cross sum_j (w_j/den_j) (y_j - x)), since x cross (.) is linear and x cross x = 0,
// which saves the per-pair cross product.
//
// FP32 kernels use 1 - x.y = |x - y|^2 / 2 for points on the sphere (no cancellation for close
// pairs), accumulate sum_j (2 w_j / (r_j^2 + 2 delta^2)) (x - y_j) in FP32 over one shared-memory
// tile and add each tile's partial into FP64 accumulators (a compensated two-level sum); the
// final u = -mult * (x cross D) uses the FP64 target position.
#include "lpm_internal.h"

#include <cmath>

namespace lpm {

namespace {

constexpr double kPi = 3.14159265358979323846264338327950288;
constexpr double kZeroTol = 1.0e-13;  // ZERO_TOL (src/LpmTypeDefs.h:33-34)

// Reciprocal: hardware approximation refined by two Newton-Raphson steps r <- r + r(1 - d r)
// (quadratic convergence from ~2^-22 gives full double precision, within one ulp).
__device__ __forceinline__ double rcp64(double d) {
    double r;
    asm("rcp.approx.ftz.f64 %0, %1;" : "=d"(r) : "d"(d));
    double e = fma(-d, r, 1.0);
    r = fma(r, e, r);
    e = fma(-d, r, 1.0);
    return fma(r, e, r);
}

// Reciprocal square root: hardware approximation refined by two Newton-Raphson steps
// y <- y + (y/2)(1 - a y^2).
__device__ __forceinline__ double rsqrt64(double a) {
    double y;
    asm("rsqrt.approx.ftz.f64 %0, %1;" : "=d"(y) : "d"(a));
    double t = a * y;
    double e = fma(-t, y, 1.0);
    y = fma(0.5 * y, e, y);
    t = a * y;
    e = fma(-t, y, 1.0);
    return fma(0.5 * y, e, y);
}

__device__ __forceinline__ float rcp32(float x) {
    float r;
    asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
    return r;
}
__device__ __forceinline__ float rsqrt32(float x) {
    float r;
    asm("rsqrt.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
    return r;
}

constexpr int kThreads = 256;
constexpr int kTile = 256;
constexpr int kTpt64 = 2;

// ------------------------------------------------------------------ FP64 Biot-Savart
template <bool kDelta>
__global__ void __launch_bounds__(kThreads) bs_f64_kernel(const double4* __restrict__ src, int64_t n_src,
                                                          const double4* __restrict__ tgt, int64_t n_tgt, double r2,
                                                          double d2, double mult, double* __restrict__ out,
                                                          int64_t stride) {
    __shared__ double4 tile[kTile];
    const int64_t base = (int64_t)blockIdx.x * (kThreads * kTpt64) + threadIdx.x;
    double tx[kTpt64], ty[kTpt64], tz[kTpt64], sx[kTpt64], sy[kTpt64], sz[kTpt64];
#pragma unroll
    for (int t = 0; t < kTpt64; ++t) {
        const int64_t i = base + t * kThreads;
        const double4 p = i < n_tgt ? tgt[i] : make_double4(0.0, 0.0, 0.0, 0.0);
        tx[t] = p.x; ty[t] = p.y; tz[t] = p.z;
        sx[t] = 0.0; sy[t] = 0.0; sz[t] = 0.0;
    }
    for (int64_t j0 = 0; j0 < n_src; j0 += kTile) {
        __syncthreads();
        const int64_t j = j0 + threadIdx.x;
        tile[threadIdx.x] = j < n_src ? src[j] : make_double4(0.0, 0.0, 0.0, 0.0);
        __syncthreads();
        const int m = (int)min((int64_t)kTile, n_src - j0);
#pragma unroll 4
        for (int k = 0; k < m; ++k) {
            const double4 s = tile[k];
#pragma unroll
            for (int t = 0; t < kTpt64; ++t) {
                // (x*x' + y*y') + z*z' rounded exactly like XyzVector::dotProduct in the reference (no
                // fused multiply-add), so den carries the same rounding error for close pairs
                const double dot = __dadd_rn(__dadd_rn(__dmul_rn(tx[t], s.x), __dmul_rn(ty[t], s.y)),
                                             __dmul_rn(tz[t], s.z));
                double den = r2 - dot;
                if (kDelta) den += d2;
                double f = s.w * rcp64(den);
                f = fabs(den) > kZeroTol ? f : 0.0;
                // x cross y = x cross (y - x): accumulating (y - x) keeps the terms at the size of
                // their cross products, so the final x cross S loses no digits to cancellation
                sx[t] = fma(f, s.x - tx[t], sx[t]);
                sy[t] = fma(f, s.y - ty[t], sy[t]);
                sz[t] = fma(f, s.z - tz[t], sz[t]);
            }
        }
    }
#pragma unroll
    for (int t = 0; t < kTpt64; ++t) {
        const int64_t i = base + t * kThreads;
        if (i < n_tgt) {
            out[i] = mult * (ty[t] * sz[t] - tz[t] * sy[t]);
            out[stride + i] = mult * (tz[t] * sx[t] - tx[t] * sz[t]);
            out[2 * stride + i] = mult * (tx[t] * sy[t] - ty[t] * sx[t]);
        }
    }
}

// ------------------------------------------------------------------ FP64 Poisson 1/(4 pi r)
__global__ void __launch_bounds__(kThreads) poisson_f64_kernel(const double4* __restrict__ src, int64_t n_src,
                                                               const double4* __restrict__ tgt, int64_t n_tgt,
                                                               double mult, double* __restrict__ out) {
    __shared__ double4 tile[kTile];
    const int64_t base = (int64_t)blockIdx.x * (kThreads * kTpt64) + threadIdx.x;
    double tx[kTpt64], ty[kTpt64], tz[kTpt64], phi[kTpt64];
#pragma unroll
    for (int t = 0; t < kTpt64; ++t) {
        const int64_t i = base + t * kThreads;
        const double4 p = i < n_tgt ? tgt[i] : make_double4(0.0, 0.0, 0.0, 0.0);
        tx[t] = p.x; ty[t] = p.y; tz[t] = p.z;
        phi[t] = 0.0;
    }
    for (int64_t j0 = 0; j0 < n_src; j0 += kTile) {
        __syncthreads();
        const int64_t j = j0 + threadIdx.x;
        tile[threadIdx.x] = j < n_src ? src[j] : make_double4(0.0, 0.0, 0.0, 0.0);
        __syncthreads();
        const int m = (int)min((int64_t)kTile, n_src - j0);
#pragma unroll 4
        for (int k = 0; k < m; ++k) {
            const double4 s = tile[k];
#pragma unroll
            for (int t = 0; t < kTpt64; ++t) {
                const double dx = tx[t] - s.x, dy = ty[t] - s.y, dz = tz[t] - s.z;
                const double rr = dx * dx + dy * dy + dz * dz;
                const double inv = rr > 0.0 ? rsqrt64(rr) : 0.0;
                phi[t] = fma(s.w, inv, phi[t]);
            }
        }
    }
#pragma unroll
    for (int t = 0; t < kTpt64; ++t) {
        const int64_t i = base + t * kThreads;
        if (i < n_tgt) out[i] = mult * phi[t];
    }
}

// ------------------------------------------------------------------ FP64 scalar kernels of the ScalarKernel family
// Pair values without the constant factor (applied once per target as `mult`), each formed as the
// reference forms it (products and sums without contraction where the reference has no FMA):
//   SphereGreensFn        -log(R^2 - y.x) / (4 pi R)           (src/LpmScalarKernel.h:31-45)
//   PlanarGreens...       log(|x - y|^2) / (4 pi)              (src/LpmScalarKernel.h:19-29)
//   SecondOrderDelta3d    3 exp(-(|x - y|/eps)^3) / (4 pi eps^3) (src/LpmScalarKernel.h:47-62)
//   SphereDelta           (2 eps^2 d - (1 - d)^2) / (4 pi (1 - d + eps^2)^2) - 1/(4 pi), d = x.y
//                                                               (src/LpmScalarKernel.h:64-78)
struct SphereGreensPair {
    double r2;
    __device__ double operator()(double tx, double ty, double tz, double sx, double sy, double sz) const {
        const double dot = __dadd_rn(__dadd_rn(__dmul_rn(sx, tx), __dmul_rn(sy, ty)), __dmul_rn(sz, tz));
        return log(r2 - dot);
    }
};
struct PlanarLogPair {
    __device__ double operator()(double tx, double ty, double tz, double sx, double sy, double sz) const {
        const double dx = tx - sx, dy = ty - sy, dz = tz - sz;
        return log(__dadd_rn(__dadd_rn(__dmul_rn(dx, dx), __dmul_rn(dy, dy)), __dmul_rn(dz, dz)));
    }
};
struct Delta3dPair {
    double inv_eps;
    __device__ double operator()(double tx, double ty, double tz, double sx, double sy, double sz) const {
        const double dx = tx - sx, dy = ty - sy, dz = tz - sz;
        const double q = sqrt(__dadd_rn(__dadd_rn(__dmul_rn(dx, dx), __dmul_rn(dy, dy)), __dmul_rn(dz, dz))) * inv_eps;
        return exp(-(q * q * q));
    }
};
struct SphereDeltaPair {
    double eps2;
    __device__ double operator()(double tx, double ty, double tz, double sx, double sy, double sz) const {
        const double d = __dadd_rn(__dadd_rn(__dmul_rn(tx, sx), __dmul_rn(ty, sy)), __dmul_rn(tz, sz));
        const double numer = 2.0 * eps2 * d - (1.0 - d) * (1.0 - d);
        const double den = 1.0 - d + eps2;
        return numer / (den * den) - 1.0;
    }
};

// out[i] = mult * sum_j w_j K(x_i, y_j), skipping j == coinc_off + i for targets i < coinc_n when
// kSkipSelf (the singular kernels' self pair, excluded by index as the reference does).
template <class K, bool kSkipSelf>
__global__ void __launch_bounds__(kThreads) scalar_f64_kernel(const double4* __restrict__ src, int64_t n_src,
                                                              const double4* __restrict__ tgt, int64_t n_tgt, K kern,
                                                              double mult, double* __restrict__ out, int64_t coinc_n,
                                                              int64_t coinc_off) {
    __shared__ double4 tile[kTile];
    const int64_t base = (int64_t)blockIdx.x * (kThreads * kTpt64) + threadIdx.x;
    double tx[kTpt64], ty[kTpt64], tz[kTpt64], phi[kTpt64];
    int64_t self[kTpt64];
#pragma unroll
    for (int t = 0; t < kTpt64; ++t) {
        const int64_t i = base + t * kThreads;
        const double4 p = i < n_tgt ? tgt[i] : make_double4(0.0, 0.0, 2.0, 0.0);
        tx[t] = p.x; ty[t] = p.y; tz[t] = p.z;
        phi[t] = 0.0;
        self[t] = kSkipSelf && i < coinc_n ? coinc_off + i : -1;
    }
    for (int64_t j0 = 0; j0 < n_src; j0 += kTile) {
        __syncthreads();
        const int64_t j = j0 + threadIdx.x;
        tile[threadIdx.x] = j < n_src ? src[j] : make_double4(0.0, 0.0, 0.0, 0.0);
        __syncthreads();
        const int m = (int)min((int64_t)kTile, n_src - j0);
        for (int k = 0; k < m; ++k) {
            const double4 s = tile[k];
#pragma unroll
            for (int t = 0; t < kTpt64; ++t) {
                if (kSkipSelf && j0 + k == self[t]) continue;
                phi[t] = fma(s.w, kern(tx[t], ty[t], tz[t], s.x, s.y, s.z), phi[t]);
            }
        }
    }
#pragma unroll
    for (int t = 0; t < kTpt64; ++t) {
        const int64_t i = base + t * kThreads;
        if (i < n_tgt) out[i] = mult * phi[t];
    }
}

template <class K>
int launch_scalar_f64(lpm_ctx* ctx, const char* name, K kern, bool skip_self, const double4* src, int64_t n_src,
                      const double4* tgt, int64_t n_tgt, double mult, double* out, int64_t coinc_n,
                      int64_t coinc_off) {
    const unsigned grid = grid_for(n_tgt, kThreads * kTpt64);
    if (skip_self)
        LPM_LAUNCH(ctx, name, (scalar_f64_kernel<K, true>), grid, kThreads, 0, src, n_src, tgt, n_tgt, kern, mult, out,
                   coinc_n, coinc_off);
    else
        LPM_LAUNCH(ctx, name, (scalar_f64_kernel<K, false>), grid, kThreads, 0, src, n_src, tgt, n_tgt, kern, mult, out,
                   coinc_n, coinc_off);
    return LPM_OK;
}

// ------------------------------------------------------------------ FP32 Biot-Savart
// src.w holds 2*strength.  Coincident (target, source) pairs -- a face-centroid target and its
// own source -- can only sit at equal indices (see coinc_* arguments); tiles that may contain one
// run the guarded loop, all others the unguarded one.
template <bool kGuard, bool kDelta, int TPT>
__device__ __forceinline__ void bs_f32_tile(const float4* tile, int m, const float* tx, const float* ty,
                                            const float* tz, float* ax, float* ay, float* az, float d2x2) {
    // Targets go in pairs through packed FMAs (fma.rn.f32x2); each lane rounds as the scalar form
    // d = t - s, rr = fma(dz, dz, fma(dy, dy, dx dx)), f = w / rr, a += f d:  t - s is fma(s, -1, t) and
    // a product is fma(a, b, -0), both exact restatements of the single-rounded operation.
    static_assert(TPT % 2 == 0, "targets are processed in pairs");
#pragma unroll 4
    for (int k = 0; k < m; ++k) {
        const float4 s = tile[k];
#pragma unroll
        for (int t = 0; t < TPT; t += 2) {
            float dx0, dx1, dy0, dy1, dz0, dz1, r0, r1, f0, f1;
            fma2p(dx0, dx1, s.x, s.x, -1.0f, tx[t], tx[t + 1]);
            fma2p(dy0, dy1, s.y, s.y, -1.0f, ty[t], ty[t + 1]);
            fma2p(dz0, dz1, s.z, s.z, -1.0f, tz[t], tz[t + 1]);
            fma2v(r0, r1, dx0, dx1, dx0, dx1, -0.0f, -0.0f);
            fma2v(r0, r1, dy0, dy1, dy0, dy1, r0, r1);
            fma2v(r0, r1, dz0, dz1, dz0, dz1, r0, r1);
            if (kDelta) { r0 += d2x2; r1 += d2x2; }
            float i0 = rcp32(r0), i1 = rcp32(r1);
            if (kGuard) {
                i0 = r0 > 2.0e-13f ? i0 : 0.0f;
                i1 = r1 > 2.0e-13f ? i1 : 0.0f;
            }
            fma2p(f0, f1, i0, i1, s.w, -0.0f, -0.0f);
            fma2v(ax[t], ax[t + 1], f0, f1, dx0, dx1, ax[t], ax[t + 1]);
            fma2v(ay[t], ay[t + 1], f0, f1, dy0, dy1, ay[t], ay[t + 1]);
            fma2v(az[t], az[t + 1], f0, f1, dz0, dz1, az[t], az[t + 1]);
        }
    }
}

// TPT targets per thread (2, 4 or 8; the context's "direct_targets"), kThreads x TPT targets per block.
template <bool kDelta, int TPT>
__global__ void __launch_bounds__(kThreads) bs_f32_kernel(const float4* __restrict__ src, int64_t n_src,
                                                          const float4* __restrict__ tgt,
                                                          const double4* __restrict__ tgt64, int64_t n_tgt,
                                                          float d2x2, double mult, double* __restrict__ out,
                                                          int64_t stride, int64_t coinc_n, int64_t coinc_off,
                                                          int64_t src_part) {
    __shared__ float4 tile[kTile];
    const int64_t blk0 = (int64_t)blockIdx.x * (kThreads * TPT);
    const int64_t base = blk0 + threadIdx.x;
    float tx[TPT], ty[TPT], tz[TPT], ax[TPT], ay[TPT], az[TPT];
    double Dx[TPT], Dy[TPT], Dz[TPT];
#pragma unroll
    for (int t = 0; t < TPT; ++t) {
        const int64_t i = base + t * kThreads;
        const float4 p = i < n_tgt ? tgt[i] : make_float4(0.f, 0.f, 0.f, 0.f);
        tx[t] = p.x; ty[t] = p.y; tz[t] = p.z;
        Dx[t] = 0.0; Dy[t] = 0.0; Dz[t] = 0.0;
    }
    // source indices that may coincide with this block's targets
    const int64_t c_lo = blk0 < coinc_n ? blk0 + coinc_off : INT64_MAX;
    const int64_t c_hi = blk0 < coinc_n ? min(blk0 + kThreads * TPT, coinc_n) + coinc_off : INT64_MIN;
    // gridDim.y source parts of src_part sources each (a multiple of kTile): blockIdx.y sums its part
    const int64_t j_begin = (int64_t)blockIdx.y * src_part, j_end = min(n_src, j_begin + src_part);
    for (int64_t j0 = j_begin; j0 < j_end; j0 += kTile) {
        __syncthreads();
        const int64_t j = j0 + threadIdx.x;
        tile[threadIdx.x] = j < j_end ? src[j] : make_float4(0.f, 0.f, 0.f, 0.f);
        __syncthreads();
        const int m = (int)min((int64_t)kTile, j_end - j0);
#pragma unroll
        for (int t = 0; t < TPT; ++t) { ax[t] = 0.f; ay[t] = 0.f; az[t] = 0.f; }
        if (j0 < c_hi && j0 + m > c_lo)
            bs_f32_tile<true, kDelta, TPT>(tile, m, tx, ty, tz, ax, ay, az, d2x2);
        else
            bs_f32_tile<false, kDelta, TPT>(tile, m, tx, ty, tz, ax, ay, az, d2x2);
#pragma unroll
        for (int t = 0; t < TPT; ++t) { Dx[t] += ax[t]; Dy[t] += ay[t]; Dz[t] += az[t]; }
    }
#pragma unroll
    for (int t = 0; t < TPT; ++t) {
        const int64_t i = base + t * kThreads;
        if (i < n_tgt) {
            const double4 p = tgt64[i];
            const double nm = -mult;
            const double u0 = nm * (p.y * Dz[t] - p.z * Dy[t]), u1 = nm * (p.z * Dx[t] - p.x * Dz[t]),
                         u2 = nm * (p.x * Dy[t] - p.y * Dx[t]);
            if (gridDim.y == 1) {
                out[i] = u0;
                out[stride + i] = u1;
                out[2 * stride + i] = u2;
            } else {  // two parts added onto a zeroed output: 0 + a + b == 0 + b + a, so the result is exact
                atomicAdd(out + i, u0);
                atomicAdd(out + stride + i, u1);
                atomicAdd(out + 2 * stride + i, u2);
            }
        }
    }
}

// ------------------------------------------------------------------ FP32 Poisson
template <bool kGuard, int TPT>
__device__ __forceinline__ void poisson_f32_tile(const float4* tile, int m, const float* tx, const float* ty,
                                                 const float* tz, float* acc) {
    // targets in pairs through packed FMAs, rounded as the scalar form (see bs_f32_tile)
#pragma unroll 4
    for (int k = 0; k < m; ++k) {
        const float4 s = tile[k];
#pragma unroll
        for (int t = 0; t < TPT; t += 2) {
            float dx0, dx1, dy0, dy1, dz0, dz1, r0, r1;
            fma2p(dx0, dx1, s.x, s.x, -1.0f, tx[t], tx[t + 1]);
            fma2p(dy0, dy1, s.y, s.y, -1.0f, ty[t], ty[t + 1]);
            fma2p(dz0, dz1, s.z, s.z, -1.0f, tz[t], tz[t + 1]);
            fma2v(r0, r1, dx0, dx1, dx0, dx1, -0.0f, -0.0f);
            fma2v(r0, r1, dy0, dy1, dy0, dy1, r0, r1);
            fma2v(r0, r1, dz0, dz1, dz0, dz1, r0, r1);
            float i0 = rsqrt32(r0), i1 = rsqrt32(r1);
            if (kGuard) {
                i0 = r0 > 0.0f ? i0 : 0.0f;
                i1 = r1 > 0.0f ? i1 : 0.0f;
            }
            fma2p(acc[t], acc[t + 1], i0, i1, s.w, acc[t], acc[t + 1]);
        }
    }
}

template <int TPT>
__global__ void __launch_bounds__(kThreads) poisson_f32_kernel(const float4* __restrict__ src, int64_t n_src,
                                                               const float4* __restrict__ tgt, int64_t n_tgt,
                                                               double mult, double* __restrict__ out, int64_t coinc_n,
                                                               int64_t coinc_off, int64_t src_part) {
    __shared__ float4 tile[kTile];
    const int64_t blk0 = (int64_t)blockIdx.x * (kThreads * TPT);
    const int64_t base = blk0 + threadIdx.x;
    float tx[TPT], ty[TPT], tz[TPT], acc[TPT];
    double phi[TPT];
#pragma unroll
    for (int t = 0; t < TPT; ++t) {
        const int64_t i = base + t * kThreads;
        const float4 p = i < n_tgt ? tgt[i] : make_float4(0.f, 0.f, 0.f, 0.f);
        tx[t] = p.x; ty[t] = p.y; tz[t] = p.z;
        phi[t] = 0.0;
    }
    const int64_t c_lo = blk0 < coinc_n ? blk0 + coinc_off : INT64_MAX;
    const int64_t c_hi = blk0 < coinc_n ? min(blk0 + kThreads * TPT, coinc_n) + coinc_off : INT64_MIN;
    const int64_t j_begin = (int64_t)blockIdx.y * src_part, j_end = min(n_src, j_begin + src_part);
    for (int64_t j0 = j_begin; j0 < j_end; j0 += kTile) {
        __syncthreads();
        const int64_t j = j0 + threadIdx.x;
        tile[threadIdx.x] = j < j_end ? src[j] : make_float4(0.f, 0.f, 0.f, 0.f);
        __syncthreads();
        const int m = (int)min((int64_t)kTile, j_end - j0);
#pragma unroll
        for (int t = 0; t < TPT; ++t) acc[t] = 0.f;
        if (j0 < c_hi && j0 + m > c_lo)
            poisson_f32_tile<true, TPT>(tile, m, tx, ty, tz, acc);
        else
            poisson_f32_tile<false, TPT>(tile, m, tx, ty, tz, acc);
#pragma unroll
        for (int t = 0; t < TPT; ++t) phi[t] += acc[t];
    }
#pragma unroll
    for (int t = 0; t < TPT; ++t) {
        const int64_t i = base + t * kThreads;
        if (i < n_tgt) {
            if (gridDim.y == 1) out[i] = mult * phi[t];
            else atomicAdd(out + i, mult * phi[t]);  // two parts onto zero: exact in either order
        }
    }
}

__global__ void pack_f32_kernel(const double4* __restrict__ in, int64_t n, float4* __restrict__ out, float wscale) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) {
        const double4 p = in[i];
        out[i] = make_float4((float)p.x, (float)p.y, (float)p.z, (float)(p.w * wscale));
    }
}

}  // namespace

int pack_f32(lpm_ctx* ctx, const double4* in, int64_t n, float4* out, bool scale_w2) {
    if (n <= 0) return LPM_OK;
    LPM_LAUNCH(ctx, "pack_f32_kernel", pack_f32_kernel, grid_for(n, 256), 256, 0, in, n, out,
               scale_w2 ? 2.0f : 1.0f);
    return LPM_OK;
}

int direct_sum_f64(lpm_ctx* ctx, const lpm_kernel_desc& k, const double4* src, int64_t n_src, const double4* tgt,
                   int64_t n_tgt, double* out, int64_t out_stride, int64_t coinc_n, int64_t coinc_off) {
    if (n_tgt <= 0) return LPM_OK;
    const unsigned grid = grid_for(n_tgt, kThreads * kTpt64);
    if (k.kind == LPM_KERNEL_BIOT_SAVART_SPHERE) {
        const double mult = -1.0 / (4.0 * kPi * k.radius);
        const double r2 = k.radius * k.radius, d2 = k.delta * k.delta;
        if (k.delta != 0.0)
            LPM_LAUNCH(ctx, "bs_f64_kernel", bs_f64_kernel<true>, grid, kThreads, 0, src, n_src, tgt, n_tgt, r2, d2, mult, out,
                                                                    out_stride);
        else
            LPM_LAUNCH(ctx, "bs_f64_kernel", bs_f64_kernel<false>, grid, kThreads, 0, src, n_src, tgt, n_tgt, r2, d2, mult, out,
                                                                     out_stride);
    } else if (k.kind == LPM_KERNEL_POISSON_3D) {
        LPM_LAUNCH(ctx, "poisson_f64_kernel", poisson_f64_kernel, grid, kThreads, 0, src, n_src, tgt, n_tgt, 1.0 / (4.0 * kPi), out);
    } else if (k.kind == LPM_KERNEL_SPHERE_GREENS) {
        return launch_scalar_f64(ctx, "scalar_f64_kernel", SphereGreensPair{k.radius * k.radius}, true, src, n_src, tgt,
                                 n_tgt, -1.0 / (4.0 * kPi * k.radius), out, coinc_n, coinc_off);
    } else if (k.kind == LPM_KERNEL_PLANAR_LOG) {
        return launch_scalar_f64(ctx, "scalar_f64_kernel", PlanarLogPair{}, true, src, n_src, tgt, n_tgt,
                                 1.0 / (4.0 * kPi), out, coinc_n, coinc_off);
    } else if (k.kind == LPM_KERNEL_DELTA_3D) {
        const double e3 = k.delta * k.delta * k.delta;
        return launch_scalar_f64(ctx, "scalar_f64_kernel", Delta3dPair{1.0 / k.delta}, false, src, n_src, tgt, n_tgt,
                                 3.0 / (4.0 * kPi * e3), out, 0, 0);
    } else if (k.kind == LPM_KERNEL_SPHERE_DELTA) {
        return launch_scalar_f64(ctx, "scalar_f64_kernel", SphereDeltaPair{k.delta * k.delta}, false, src, n_src, tgt,
                                 n_tgt, 1.0 / (4.0 * kPi), out, 0, 0);
    } else {
        set_error("invalid kernel");
        return LPM_ERR_KERNEL;
    }
    return LPM_OK;
}

// FP32 sums take FP32 copies of sources (w pre-scaled by 2 for Biot-Savart) and targets, plus the
// FP64 targets for the Biot-Savart epilogue.  Targets 0..coinc_n-1 may coincide with sources
// coinc_off..coinc_off+coinc_n-1 (face-centroid targets and their own sources).
namespace {
// Source parts of an FP32 direct sum: the target blocks alone may fill their last wave of resident blocks
// poorly (at 3 resident 256-thread blocks per SM, 1,920 blocks are 4.3 waves on 148 SMs, the fifth a third
// full).  Splitting the sources in two halves doubles the blocks at half the work each; the split is taken
// when it shortens the estimate ceil(blocks parts / resident) / parts.  Two parts only: two addends onto
// a zeroed output are exact in either order, so the result does not depend on which part finishes first.
template <typename Kern>
int source_parts(lpm_ctx* ctx, Kern kern, int64_t blocks, int64_t n_src) {
    int per_sm = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, kThreads, 0) != cudaSuccess || per_sm < 1)
        return 1;
    const double resident = (double)per_sm * ctx->num_sms;
    if (n_src < 2 * kTile) return 1;
    const double t1 = std::ceil(blocks / resident), t2 = std::ceil(2.0 * blocks / resident) / 2.0;
    return t2 < t1 ? 2 : 1;
}
}  // namespace

template <int TPT>
static int direct_sum_f32_tpt(lpm_ctx* ctx, const lpm_kernel_desc& k, const float4* src, int64_t n_src,
                              const float4* tgt, const double4* tgt64, int64_t n_tgt, double* out, int64_t out_stride,
                              int64_t coinc_n, int64_t coinc_off);

int direct_sum_f32_impl(lpm_ctx* ctx, const lpm_kernel_desc& k, const float4* src, int64_t n_src, const float4* tgt,
                        const double4* tgt64, int64_t n_tgt, double* out, int64_t out_stride, int64_t coinc_n,
                        int64_t coinc_off) {
    switch (ctx->direct_tpt) {
        case 2: return direct_sum_f32_tpt<2>(ctx, k, src, n_src, tgt, tgt64, n_tgt, out, out_stride, coinc_n, coinc_off);
        case 8: return direct_sum_f32_tpt<8>(ctx, k, src, n_src, tgt, tgt64, n_tgt, out, out_stride, coinc_n, coinc_off);
        default:
            return direct_sum_f32_tpt<4>(ctx, k, src, n_src, tgt, tgt64, n_tgt, out, out_stride, coinc_n, coinc_off);
    }
}

template <int TPT>
static int direct_sum_f32_tpt(lpm_ctx* ctx, const lpm_kernel_desc& k, const float4* src, int64_t n_src,
                              const float4* tgt, const double4* tgt64, int64_t n_tgt, double* out, int64_t out_stride,
                              int64_t coinc_n, int64_t coinc_off) {
    if (n_tgt <= 0) return LPM_OK;
    const unsigned grid = grid_for(n_tgt, kThreads * TPT);
    auto zero_rows = [&](int rows) -> int {
        for (int c = 0; c < rows; ++c)
            LPM_CUDA_TRY(cudaMemsetAsync(out + (size_t)c * out_stride, 0, sizeof(double) * (size_t)n_tgt, ctx->stream));
        return LPM_OK;
    };
    if (k.kind == LPM_KERNEL_BIOT_SAVART_SPHERE) {
        const double mult = -1.0 / (4.0 * kPi * k.radius);
        const bool delta = k.delta != 0.0;
        const int parts = delta ? source_parts(ctx, bs_f32_kernel<true, TPT>, grid, n_src)
                                : source_parts(ctx, bs_f32_kernel<false, TPT>, grid, n_src);
        const int64_t part = parts == 1 ? n_src : ((n_src + 2 * kTile - 1) / (2 * kTile)) * kTile;
        if (parts > 1) {
            int rc = zero_rows(3);
            if (rc) return rc;
        }
        const dim3 g(grid, parts);
        if (delta)
            LPM_LAUNCH(ctx, "bs_f32_kernel", (bs_f32_kernel<true, TPT>), g, kThreads, 0, src, n_src, tgt, tgt64, n_tgt,
                       (float)(2.0 * k.delta * k.delta), mult, out, out_stride, coinc_n, coinc_off, part);
        else
            LPM_LAUNCH(ctx, "bs_f32_kernel", (bs_f32_kernel<false, TPT>), g, kThreads, 0, src, n_src, tgt, tgt64, n_tgt, 0.0f,
                       mult, out, out_stride, coinc_n, coinc_off, part);
    } else if (k.kind == LPM_KERNEL_POISSON_3D) {
        const int parts = source_parts(ctx, poisson_f32_kernel<TPT>, grid, n_src);
        const int64_t part = parts == 1 ? n_src : ((n_src + 2 * kTile - 1) / (2 * kTile)) * kTile;
        if (parts > 1) {
            int rc = zero_rows(1);
            if (rc) return rc;
        }
        const dim3 g(grid, parts);
        LPM_LAUNCH(ctx, "poisson_f32_kernel", poisson_f32_kernel<TPT>, g, kThreads, 0, src, n_src, tgt, n_tgt,
                   1.0 / (4.0 * kPi), out, coinc_n, coinc_off, part);
    } else {
        set_error("invalid kernel");
        return LPM_ERR_KERNEL;
    }
    return LPM_OK;
}

int check_kernel_desc(const lpm_kernel_desc* k) {
    if (!k) {
        set_error("null kernel descriptor");
        return LPM_ERR_ARG;
    }
    if (k->kind < LPM_KERNEL_BIOT_SAVART_SPHERE || k->kind > LPM_KERNEL_SPHERE_DELTA) {
        set_error("invalid kernel");
        return LPM_ERR_KERNEL;
    }
    if ((k->kind == LPM_KERNEL_BIOT_SAVART_SPHERE || k->kind == LPM_KERNEL_SPHERE_GREENS) && !(k->radius > 0.0)) {
        set_error("sphere kernels need radius > 0");
        return LPM_ERR_ARG;
    }
    if ((k->kind == LPM_KERNEL_DELTA_3D || k->kind == LPM_KERNEL_SPHERE_DELTA) && !(k->delta > 0.0)) {
        set_error("delta kernels need eps (the delta field) > 0");
        return LPM_ERR_ARG;
    }
    return LPM_OK;
}

// The FP32 direct sums exist for the Biot-Savart and 3D Poisson kernels only; every FP32 entry point checks
// this before it launches anything.
int check_f32_kind(const lpm_kernel_desc& k) {
    if (k.kind != LPM_KERNEL_BIOT_SAVART_SPHERE && k.kind != LPM_KERNEL_POISSON_3D) {
        set_error("invalid kernel: the FP32 direct sum takes the Biot-Savart and 3D Poisson kernels (use LPM_PREC_F64)");
        return LPM_ERR_KERNEL;
    }
    return LPM_OK;
}

// Device entry shared by the C ABI: FP64 or FP32 (FP32 copies go to scratch slots).
int direct_sum_any(lpm_ctx* ctx, const lpm_kernel_desc& k, int precision, const double4* src, int64_t n_src,
                   const double4* tgt, int64_t n_tgt, double* out, int64_t coinc_n, int64_t coinc_off) {
    if (precision == LPM_PREC_F64) return direct_sum_f64(ctx, k, src, n_src, tgt, n_tgt, out, n_tgt, coinc_n, coinc_off);
    if (precision != LPM_PREC_F32) {
        set_error("unknown precision %d", precision);
        return LPM_ERR_ARG;
    }
    int rc = check_f32_kind(k);
    if (rc) return rc;
    float4* s32 = (float4*)scratch(ctx, kSlotSrc32, sizeof(float4) * (size_t)std::max<int64_t>(n_src, 1));
    float4* t32 = (float4*)scratch(ctx, kSlotTgt32, sizeof(float4) * (size_t)std::max<int64_t>(n_tgt, 1));
    if (!s32 || !t32) return LPM_ERR_OOM;
    rc = pack_f32(ctx, src, n_src, s32, k.kind == LPM_KERNEL_BIOT_SAVART_SPHERE);
    if (rc) return rc;
    rc = pack_f32(ctx, tgt, n_tgt, t32, false);
    if (rc) return rc;
    return direct_sum_f32_impl(ctx, k, s32, n_src, t32, tgt, n_tgt, out, n_tgt, coinc_n, coinc_off);
}

}  // namespace lpm

using namespace lpm;

extern "C" int lpm_direct_sum_dev(lpm_ctx* ctx, const lpm_kernel_desc* kernel, int precision, const double* src,
                                  int64_t n_src, const double* tgt, int64_t n_tgt, int64_t n_coincident,
                                  double* out) {
    if (!ctx) {
        set_error("null context");
        return LPM_ERR_ARG;
    }
    int rc = check_kernel_desc(kernel);
    if (rc) return rc;
    if (n_src < 0 || n_tgt < 0 || (n_src > 0 && !src) || (n_tgt > 0 && (!tgt || !out)) || n_coincident < 0 ||
        n_coincident > std::min(n_src, n_tgt)) {
        set_error("lpm_direct_sum_dev: bad sizes or null pointers");
        return LPM_ERR_ARG;
    }
    LPM_CUDA_TRY(cudaSetDevice(ctx->device));
    return direct_sum_any(ctx, *kernel, precision, (const double4*)src, n_src, (const double4*)tgt, n_tgt, out,
                          n_coincident, 0);
}

extern "C" int lpm_direct_sum_mesh(lpm_ctx* ctx, const lpm_kernel_desc* kernel, int precision, int64_t n_verts,
                                   const double* vx, const double* vy, const double* vz, int64_t n_faces,
                                   const double* fx, const double* fy, const double* fz, const double* face_area,
                                   const uint8_t* face_divided, const double* face_src, int64_t vert_begin,
                                   int64_t vert_end, int64_t face_begin, int64_t face_end, double* vert_out0,
                                   double* vert_out1, double* vert_out2, double* face_out0, double* face_out1,
                                   double* face_out2) {
    if (!ctx) {
        set_error("null context");
        return LPM_ERR_ARG;
    }
    int rc = check_kernel_desc(kernel);
    if (rc) return rc;
    const bool vec = kernel->kind == LPM_KERNEL_BIOT_SAVART_SPHERE;
    const int comps = vec ? 3 : 1;
    if (n_verts < 0 || n_faces < 0 || (n_verts > 0 && (!vx || !vy || !vz)) ||
        (n_faces > 0 && (!fx || !fy || !fz || !face_area || !face_divided || !face_src))) {
        set_error("lpm_direct_sum_mesh: null input arrays");
        return LPM_ERR_ARG;
    }
    // empty ranges (end < begin) are allowed, as for a rank with no items
    const bool do_v = vert_end >= vert_begin, do_f = face_end >= face_begin;
    if ((do_v && (vert_begin < 0 || vert_end >= n_verts || !vert_out0 || (vec && (!vert_out1 || !vert_out2)))) ||
        (do_f && (face_begin < 0 || face_end >= n_faces || !face_out0 || (vec && (!face_out1 || !face_out2))))) {
        set_error("lpm_direct_sum_mesh: target range out of bounds or null outputs");
        return LPM_ERR_ARG;
    }
    LPM_CUDA_TRY(cudaSetDevice(ctx->device));
    // sources: undivided faces in index order; face targets: undivided faces in [face_begin, face_end]
    int64_t n_src = 0, src_before_fb = 0, n_ft = 0;
    for (int64_t i = 0; i < n_faces; ++i) {
        if (!face_divided[i]) {
            if (i < face_begin) ++src_before_fb;
            if (do_f && i >= face_begin && i <= face_end) ++n_ft;
            ++n_src;
        }
    }
    const int64_t n_vt = do_v ? vert_end - vert_begin + 1 : 0;
    const int64_t n_tgt = n_ft + n_vt;
    const size_t in_bytes = sizeof(double4) * (size_t)(n_src + n_tgt);
    const size_t out_bytes = sizeof(double) * comps * (size_t)n_tgt;
    double* host = (double*)pinned(ctx, in_bytes + out_bytes);
    if (!host) return LPM_ERR_OOM;
    double4* hsrc = (double4*)host;
    double4* htgt = hsrc + n_src;
    double* hout = (double*)(htgt + n_tgt);
    int64_t s = 0, t = 0;
    for (int64_t i = 0; i < n_faces; ++i) {
        if (face_divided[i]) continue;
        hsrc[s++] = make_double4(fx[i], fy[i], fz[i], face_src[i] * face_area[i]);
        if (do_f && i >= face_begin && i <= face_end) htgt[t++] = make_double4(fx[i], fy[i], fz[i], 0.0);
    }
    for (int64_t i = 0; i < n_vt; ++i) {
        const int64_t v = vert_begin + i;
        htgt[t++] = make_double4(vx[v], vy[v], vz[v], 0.0);
    }
    double4* dsrc = (double4*)scratch(ctx, kSlotSrcPack, sizeof(double4) * (size_t)std::max<int64_t>(n_src, 1));
    double4* dtgt = (double4*)scratch(ctx, kSlotTgtPack, sizeof(double4) * (size_t)std::max<int64_t>(n_tgt, 1));
    double* dout = (double*)scratch(ctx, kSlotOut, std::max<size_t>(out_bytes, 8));
    if (!dsrc || !dtgt || !dout) return LPM_ERR_OOM;
    if (n_tgt > 0) {
        if (n_src > 0)
            LPM_CUDA_TRY(cudaMemcpyAsync(dsrc, hsrc, sizeof(double4) * (size_t)n_src, cudaMemcpyHostToDevice,
                                         ctx->stream));
        LPM_CUDA_TRY(cudaMemcpyAsync(dtgt, htgt, sizeof(double4) * (size_t)n_tgt, cudaMemcpyHostToDevice, ctx->stream));
        // face targets come first and sit on sources src_before_fb.. in order: the self pairs a singular
        // scalar kernel skips (the FP32 paths use the same indices to guard coincident pairs)
        rc = direct_sum_any(ctx, *kernel, precision, dsrc, n_src, dtgt, n_tgt, dout, n_ft, src_before_fb);
        if (rc) return rc;
        LPM_CUDA_TRY(cudaMemcpyAsync(hout, dout, out_bytes, cudaMemcpyDeviceToHost, ctx->stream));
        LPM_CUDA_TRY(cudaStreamSynchronize(ctx->stream));
    }
    t = 0;
    for (int64_t i = face_begin; do_f && i <= face_end; ++i) {
        if (face_divided[i]) continue;
        face_out0[i] = hout[t];
        if (vec) {
            face_out1[i] = hout[n_tgt + t];
            face_out2[i] = hout[2 * n_tgt + t];
        }
        ++t;
    }
    for (int64_t i = 0; i < n_vt; ++i, ++t) {
        vert_out0[vert_begin + i] = hout[t];
        if (vec) {
            vert_out1[vert_begin + i] = hout[n_tgt + t];
            vert_out2[vert_begin + i] = hout[2 * n_tgt + t];
        }
    }
    return LPM_OK;
}

extern "C" int lpm_direct_sum_meshfree(lpm_ctx* ctx, const lpm_kernel_desc* kernel, int precision, int64_t n,
                                       const double* x, const double* y, const double* z, const double* src,
                                       const double* weights, int64_t begin, int64_t end, double* out) {
    if (!ctx) {
        set_error("null context");
        return LPM_ERR_ARG;
    }
    int rc = check_kernel_desc(kernel);
    if (rc) return rc;
    if (kernel->kind == LPM_KERNEL_BIOT_SAVART_SPHERE) {
        set_error("invalid kernel: lpm_direct_sum_meshfree takes a scalar kernel");
        return LPM_ERR_KERNEL;
    }
    if (n < 0 || (n > 0 && (!x || !y || !z || !src))) {
        set_error("lpm_direct_sum_meshfree: null input arrays");
        return LPM_ERR_ARG;
    }
    const bool any = end >= begin;
    if (any && (begin < 0 || end >= n || !out)) {
        set_error("lpm_direct_sum_meshfree: target range out of bounds");
        return LPM_ERR_ARG;
    }
    if (!any || n == 0) return LPM_OK;
    LPM_CUDA_TRY(cudaSetDevice(ctx->device));
    const int64_t n_tgt = end - begin + 1;
    const size_t in_bytes = sizeof(double4) * (size_t)n;
    const size_t out_bytes = sizeof(double) * (size_t)n_tgt;
    double* host = (double*)pinned(ctx, in_bytes + out_bytes);
    if (!host) return LPM_ERR_OOM;
    double4* hsrc = (double4*)host;
    double* hout = (double*)(hsrc + n);
    for (int64_t i = 0; i < n; ++i)
        hsrc[i] = make_double4(x[i], y[i], z[i], weights ? src[i] * weights[i] : src[i]);
    double4* dsrc = (double4*)scratch(ctx, kSlotSrcPack, in_bytes);
    double* dout = (double*)scratch(ctx, kSlotOut, out_bytes);
    if (!dsrc || !dout) return LPM_ERR_OOM;
    LPM_CUDA_TRY(cudaMemcpyAsync(dsrc, hsrc, in_bytes, cudaMemcpyHostToDevice, ctx->stream));
    rc = direct_sum_any(ctx, *kernel, precision, dsrc, n, dsrc + begin, n_tgt, dout, n_tgt, begin);
    if (rc) return rc;
    LPM_CUDA_TRY(cudaMemcpyAsync(hout, dout, out_bytes, cudaMemcpyDeviceToHost, ctx->stream));
    LPM_CUDA_TRY(cudaStreamSynchronize(ctx->stream));
    for (int64_t i = 0; i < n_tgt; ++i) out[begin + i] = hout[i];
    return LPM_OK;
}
