// Treecode (TreeSum) for the spherical Biot-Savart kernel on the GPU.
//
// The reference's TreeSum (src/LpmTreeSum.cpp:55-197) is a per-target recursion over a source octree
// with Taylor moments and far-field coefficients of 1/(1 - x.y) about each box centre.  For points on
// the unit sphere 1 - x.y = |x - y|^2 / 2, so the kernel is
//     K(x, y) = (x cross y)/(1 - x.y) = 2 (x cross y) g(y),   g(y) = 1/|x - y|^2,
// and this file expands g instead: its Taylor series about a centre c converges for |y - c| < |x - c|
// (a Euclidean acceptance criterion, like the reference's box.maxRadius/|c - x| < theta at
// src/LpmTreeSum.cpp:22-24), whereas the series of 1/(1 - x.y) about a point off the sphere converges
// only inside the tangent-plane distance and its Cartesian terms cancel catastrophically for nearby
// clusters.
//
// Far field.  With d = c - x, h = y - c, e = d/|d|^2 and s = |e|^2, the generating function of the
// Chebyshev polynomials of the second kind, 1/(1 - 2tu + t^2) = sum_n U_n(u) t^n, gives
//     g(c + h) = (1/|d|^2) sum_{q,m} (-1)^m C(q+m, m) (-2)^q (e.h)^q (s |h|^2)^m,
// truncated at total degree q + 2m < P (Taylor order P, multi-indices |k| < P as SumNode's
// (src/LpmTreeSum.cpp:9-18)).  Expanding (e.h)^q = sum_{|k|=q} (q!/k!) e^k h^k turns a cluster's
// contribution into four polynomials in (e, s) whose coefficients depend on the cluster only:
//     B^0_{m,k} = (-1)^m C(|k|+m, m) (-2)^{|k|} (|k|!/k!) N_{k,m},     N_{k,m} = sum_j w_j h_j^k |h_j|^{2m},
//     B^i_{m,k} = same prefactor * N_{k+e_i,m}                          (the h_i part of y = c + h),
// evaluated per target by nested Horner schemes (4 FMAs per coefficient, a few registers live):
//     G0 = sum_j w_j g(y_j),  G_i = sum_j w_j h_ij g(y_j),
//     sum_j w_j (x cross y_j) 2 g(y_j) = 2 [ (x cross d) G0 + x cross G ].
// Moments are FP64: ordinary moments sum_j w_j h^k of every leaf from its particles, shifted to parents
// (M2M) level by level, then converted to the B coefficients.  Orders >= f64_from evaluate in FP64 (every
// order for LPM_PREC_F64 solvers, none by default for FP32 ones; run-time "f64_from"), the others in FP32,
// always accumulated in FP64.
//
// Near field.  Targets are sorted by Morton key into batches of kBatch; a batch and a source node
// interact in the far field when rho_node < theta (|x_batch - c| - r_batch), otherwise leaves interact
// directly: runs of consecutive leaves are contiguous ranges of tree-ordered sources, summed with FP32
// pair arithmetic (|x - y|^2 form, as the FP32 direct sum) and FP64 accumulation across tiles.
#include "treecode.h"

#include "mlp.h"
#include "octree.h"

#include <algorithm>
#include <cmath>
#include <new>
#include <mutex>
#include <string>
#include <vector>

namespace lpm {

namespace {

constexpr int kPMax = 12;        // highest supported Taylor order
constexpr int kBatch = 128;      // targets per batch (threads per far/near block)
constexpr int kTreeDepth = 10;   // key levels sorted for the treecode's source tree
constexpr double kPi = 3.14159265358979323846264338327950288;

__host__ __device__ constexpr int tet(int q) { return q * (q + 1) * (q + 2) / 6; }  // #{k : |k| < q}
__host__ __device__ constexpr int entries_for(int P) {                             // #{(m,k): |k| + 2m < P}
    int e = 0;
    for (int m = 0; 2 * m < P; ++m) e += tet(P - 2 * m);
    return e;
}
// The FP32 far field of the highest order runs as two launches (its fully unrolled body overflows the
// instruction cache): part 1 the Horner blocks m >= 1 times s, part 2 the block m = 0 (entries of the Horner
// sequence: part 1 first, part 2 after); part 0 is the whole sequence.
constexpr int kFarSplitOrder = 11;
__host__ __device__ constexpr int part_entries(int P, int part) {
    return part == 0 ? entries_for(P) : (part == 1 ? entries_for(P) - tet(P) : tet(P));
}
// Node moments are stored packed: the monomials (a, b, c) with a + b + c <= pm in a-major, then b, then c
// order, mono_count(pm) doubles per node.
__host__ __device__ constexpr int tet_count(int n) { return (n + 1) * (n + 2) * (n + 3) / 6; }
__host__ __device__ constexpr int mono_count(int pm) { return tet_count(pm); }
__host__ __device__ constexpr int mono_index(int a, int b, int c, int pm) {
    return tet_count(pm) - tet_count(pm - a) + b * (pm - a + 1) - b * (b - 1) / 2 + c;
}

struct CutoffTable {
    int32_t direct_below[kPMax + 1];  // a cluster with fewer sources than this is summed directly
    int32_t table_off[kPMax + 2];     // offsets of each order's gather table
};

__constant__ double c_binom[kPMax + 2][kPMax + 2];
__constant__ double c_fact[2 * kPMax + 2];

// ---------------------------------------------------------------------------------- block helpers
template <typename T>
__device__ T block_sum(T v, T* sh) {
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    const int w = threadIdx.x >> 5, lane = threadIdx.x & 31, nw = blockDim.x >> 5;
    __syncthreads();
    if (lane == 0) sh[w] = v;
    __syncthreads();
    T r = 0;
    for (int i = 0; i < nw; ++i) r += sh[i];
    return r;
}
__device__ double block_max(double v, double* sh) {
    for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
    const int w = threadIdx.x >> 5, lane = threadIdx.x & 31, nw = blockDim.x >> 5;
    __syncthreads();
    if (lane == 0) sh[w] = v;
    __syncthreads();
    double r = 0;
    for (int i = 0; i < nw; ++i) r = fmax(r, sh[i]);
    return r;
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

// ---------------------------------------------------------------------------------- per-evaluation kernels
__global__ void gather_sources_kernel(const double4* __restrict__ X, const int32_t* __restrict__ perm,
                                      const int32_t* __restrict__ counters, double4* __restrict__ out) {
    const int n = counters[0];
    for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < n; q += gridDim.x * blockDim.x) out[q] = X[perm[q]];
}

// Leaves: centre (mean position), radius, FP32 source copies (w scaled by wscale: 2 folds the factor of
// 1/(1 - x.y) = 2/|x - y|^2 of the sphere kernel into the strength) and ordinary moments
// mom[a][b][c] = sum_j w_j h^(a,b,c) for a+b+c <= pm.  A moment unit (a, b, c0) is a run of
// kP2mRun monomials (a, b, c0 .. c0 + kP2mRun - 1) (those past a + b + c = pm are computed and dropped): per
// particle its thread reads w, h_x^a, h_y^b, h_z^c0 and h_z from the power tables and walks the run by
// multiplying with h_z, five shared-memory reads for four moments.
constexpr int kP2mRun = 4;
constexpr int kP2mThreads = 128;
constexpr int kP2mUnitsPerThread = 2;
constexpr int p2m_units_for(int pm) {
    int n = 0;
    for (int a = 0; a <= pm; ++a)
        for (int b = 0; a + b <= pm; ++b) n += (pm - a - b + kP2mRun) / kP2mRun;
    return n;
}
static_assert(p2m_units_for(kPMax) <= kP2mThreads * kP2mUnitsPerThread, "leaf moment units per block");

__global__ void __launch_bounds__(kP2mThreads) leaf_p2m_kernel(Octree t, const double4* __restrict__ src, int pm,
                                                               const int4* __restrict__ units, int n_units,
                                                               double4* __restrict__ node_ctr,
                                                               double* __restrict__ node_wabs,
                                                               double* __restrict__ node_mom,
                                                               float4* __restrict__ src32, double wscale,
                                                               int heavy_cap) {
    __shared__ double sh[32];
    __shared__ double pw[32][3][kPMax + 1];
    __shared__ double ww[32];
    const int nleaves = t.counters[3];
    const int nm = mono_count(pm);
    for (int leaf = blockIdx.x; leaf < nleaves; leaf += gridDim.x) {
        const int node = t.leaf_node[leaf];
        const int s = t.node_start[node], e = t.node_end[node];
        double sx = 0, sy = 0, sz = 0, sw = 0;
        for (int q = s + threadIdx.x; q < e; q += blockDim.x) {
            const double4 p = src[q];
            sx += p.x; sy += p.y; sz += p.z; sw += fabs(p.w);
        }
        const double inv = 1.0 / (double)max(e - s, 1);
        const double cx = block_sum(sx, sh) * inv, cy = block_sum(sy, sh) * inv, cz = block_sum(sz, sh) * inv;
        const double wabs = block_sum(sw, sh);
        double r = 0;
        for (int q = s + threadIdx.x; q < e; q += blockDim.x) {
            const double4 p = src[q];
            const double hx = p.x - cx, hy = p.y - cy, hz = p.z - cz;
            r = fmax(r, sqrt(hx * hx + hy * hy + hz * hz));
            src32[q] = make_float4((float)p.x, (float)p.y, (float)p.z, (float)(wscale * p.w));
        }
        r = block_max(r, sh);
        if (threadIdx.x == 0) {
            node_ctr[node] = make_double4(cx, cy, cz, r);
            node_wabs[node] = wabs;
        }
        // moments, 32 particles at a time with their power tables in shared memory (nodes past the
        // moment capacity get none: the traversal never accepts them as far clusters)
        if (node >= heavy_cap) continue;  // uniform per block
        double acc[kP2mUnitsPerThread][kP2mRun] = {};
        for (int q0 = s; q0 < e; q0 += 32) {
            __syncthreads();
            if (threadIdx.x < 32) {
                const int q = q0 + threadIdx.x;
                double h[3] = {0, 0, 0}, w = 0;
                if (q < e) {
                    const double4 p = src[q];
                    h[0] = p.x - cx; h[1] = p.y - cy; h[2] = p.z - cz; w = p.w;
                }
                ww[threadIdx.x] = w;
                for (int a = 0; a < 3; ++a) {
                    double v = 1.0;
                    for (int k = 0; k <= pm; ++k) {
                        pw[threadIdx.x][a][k] = v;
                        v *= h[a];
                    }
                }
            }
            __syncthreads();
            const int np = min(32, e - q0);
#pragma unroll
            for (int r2 = 0; r2 < kP2mUnitsPerThread; ++r2) {
                const int u = threadIdx.x + r2 * kP2mThreads;
                if (u < n_units) {
                    const int4 k = units[u];
                    for (int j = 0; j < np; ++j) {
                        double v = ww[j] * pw[j][0][k.x] * pw[j][1][k.y] * pw[j][2][k.z];
                        const double hz = pw[j][2][1];
#pragma unroll
                        for (int c = 0; c < kP2mRun; ++c) {
                            acc[r2][c] += v;
                            v *= hz;
                        }
                    }
                }
            }
        }
        double* mout = node_mom + (size_t)node * nm;
#pragma unroll
        for (int r2 = 0; r2 < kP2mUnitsPerThread; ++r2) {
            const int u = threadIdx.x + r2 * kP2mThreads;
            if (u < n_units) {
                const int4 k = units[u];  // the run's monomials are consecutive in the packed order
                const int base = mono_index(k.x, k.y, k.z, pm);
#pragma unroll
                for (int c = 0; c < kP2mRun; ++c)
                    if (k.x + k.y + k.z + c <= pm) mout[base + c] = acc[r2][c];
            }
        }
        __syncthreads();
    }
}

// Internal nodes: centre = count-weighted mean of the children's centres, radius bound
// max(|c_child - c| + r_child), moments shifted from the children:
// m_k(c) = sum_child sum_{j <= k} C(k, j) (c_child - c)^(k-j) m_j(c_child).
// The children's moments (packed in monomial order), their shift powers and the binomial table are
// staged in shared memory, so the inner loops read no global or constant memory.
//
// One launch does the whole upward pass: pending[node] counts the internal children not yet done; a block
// starts at each internal node whose children are all leaves (their moments come from leaf_p2m_kernel), and
// the block that completes a node's last internal child goes on to the node itself (no level barriers, no
// waits).  Writers fence before the counter's decrement and the next block reads the children through L2.

// A double4 written by another block of the running launch: two 16-byte loads that skip L1.
__device__ __forceinline__ double4 ldcg4(const double4* p) {
    const double2 a = __ldcg((const double2*)p), b = __ldcg((const double2*)p + 1);
    return make_double4(a.x, a.y, b.x, b.y);
}

__global__ void m2m_pending_kernel(Octree t, int32_t* __restrict__ pending) {
    const int nn = t.counters[1];
    for (int node = blockIdx.x * blockDim.x + threadIdx.x; node < nn; node += gridDim.x * blockDim.x) {
        const int nc = t.node_nchild[node];
        int p = 0;
        for (int k = 0; k < nc; ++k) p += t.node_nchild[t.node_first_child[node] + k] > 0;
        pending[node] = p;
    }
}

constexpr int kM2mThreads = 256;
__global__ void __launch_bounds__(kM2mThreads) m2m_upward_kernel(Octree t, int pm, const int4* __restrict__ mono,
                                                         int n_mono, double4* __restrict__ node_ctr,
                                                         double* __restrict__ node_wabs,
                                                         double* __restrict__ node_mom, int heavy_cap,
                                                         int32_t* __restrict__ pending) {
    extern __shared__ double m2m_sh[];  // 2 x 8 x n_mono: child moments and their partial shifts
    __shared__ double dp[8][3][kPMax + 1];
    __shared__ double bin[kPMax + 1][kPMax + 1];
    __shared__ int mono_idx[kPMax + 1][kPMax + 1][kPMax + 1];  // (a, b, c) -> position in the monomial list
    __shared__ int climb;
    __shared__ double4 ch[8];  // the current node's children: centres (w = radius), counts, sum |w|
    __shared__ double chm[8], chw[8];
    for (int i = threadIdx.x; i < (kPMax + 1) * (kPMax + 1); i += blockDim.x)
        bin[i / (kPMax + 1)][i % (kPMax + 1)] = c_binom[i / (kPMax + 1)][i % (kPMax + 1)];
    for (int i = threadIdx.x; i < n_mono; i += blockDim.x) {
        const int4 k = mono[i];
        mono_idx[k.x][k.y][k.z] = i;
    }
    __syncthreads();
    // one internal node (block-wide); the children's centres, weights and moments were written by other
    // blocks of this launch (or by leaf_p2m_kernel) and are read past L1
    auto m2m_node = [&](int node) {
        const int nc = t.node_nchild[node];
        const int fc = t.node_first_child[node];
        __syncthreads();  // the previous node's readers of ch / dp / m2m_sh are done
        if ((int)threadIdx.x < nc) {  // the children's centres, counts and weights, one thread each
            ch[threadIdx.x] = ldcg4(node_ctr + fc + threadIdx.x);
            chm[threadIdx.x] = (double)(t.node_end[fc + threadIdx.x] - t.node_start[fc + threadIdx.x]);
            chw[threadIdx.x] = __ldcg(node_wabs + fc + threadIdx.x);
        }
        __syncthreads();
        double cx = 0, cy = 0, cz = 0, cnt = 0, wabs = 0;
        for (int k = 0; k < nc; ++k) {
            cx += chm[k] * ch[k].x; cy += chm[k] * ch[k].y; cz += chm[k] * ch[k].z; cnt += chm[k];
            wabs += chw[k];
        }
        cx /= cnt; cy /= cnt; cz /= cnt;
        double r = 0;
        for (int k = 0; k < nc; ++k) {
            const double dx = ch[k].x - cx, dy = ch[k].y - cy, dz = ch[k].z - cz;
            r = fmax(r, sqrt(dx * dx + dy * dy + dz * dz) + ch[k].w);
        }
        if (threadIdx.x == 0) {
            node_ctr[node] = make_double4(cx, cy, cz, r);
            node_wabs[node] = wabs;
        }
        if (fc + nc > heavy_cap) return;  // uniform per block: a child (numbered after node) has no moments
        if (threadIdx.x < nc * 3) {
            const int k = threadIdx.x / 3, a = threadIdx.x % 3;
            const double4 cc = ch[k];
            const double d = a == 0 ? cc.x - cx : (a == 1 ? cc.y - cy : cc.z - cz);
            double v = 1.0;
            for (int q = 0; q <= pm; ++q) {
                dp[k][a][q] = v;
                v *= d;
            }
        }
        double* S0 = m2m_sh;                  // nc x n_mono
        double* S1 = m2m_sh + 8 * n_mono;     // nc x n_mono
        const double* cm = node_mom + (size_t)fc * n_mono;  // the children are consecutive nodes
#pragma unroll 4
        for (int i = threadIdx.x; i < nc * n_mono; i += blockDim.x) S0[i] = __ldcg(cm + i);
        __syncthreads();
        // the shift factorises by axis: three 1D binomial shifts (x, then y, then z with the sum over
        // children), (k_x + 1) + (k_y + 1) + (k_z + 1) terms per monomial instead of their product
        for (int i = threadIdx.x; i < nc * n_mono; i += blockDim.x) {
            const int k = i / n_mono, term = i - k * n_mono;
            const int4 kk = mono[term];
            double acc = 0;
            for (int j0 = 0; j0 <= kk.x; ++j0)
                acc = fma(bin[kk.x][j0] * dp[k][0][kk.x - j0], S0[k * n_mono + mono_idx[j0][kk.y][kk.z]], acc);
            S1[i] = acc;
        }
        __syncthreads();
        for (int i = threadIdx.x; i < nc * n_mono; i += blockDim.x) {
            const int k = i / n_mono, term = i - k * n_mono;
            const int4 kk = mono[term];
            double acc = 0;
            for (int j1 = 0; j1 <= kk.y; ++j1)
                acc = fma(bin[kk.y][j1] * dp[k][1][kk.y - j1], S1[k * n_mono + mono_idx[kk.x][j1][kk.z]], acc);
            S0[i] = acc;
        }
        __syncthreads();
        double* mout = node_mom + (size_t)node * n_mono;
        for (int term = threadIdx.x; term < n_mono; term += blockDim.x) {
            const int4 kk = mono[term];
            double acc = 0;
            for (int k = 0; k < nc; ++k)
                for (int j2 = 0; j2 <= kk.z; ++j2)
                    acc = fma(bin[kk.z][j2] * dp[k][2][kk.z - j2], S0[k * n_mono + mono_idx[kk.x][kk.y][j2]], acc);
            mout[term] = acc;
        }
    };
    const int nn = t.counters[1];
    for (int start = blockIdx.x; start < nn; start += gridDim.x) {
        const int nc = t.node_nchild[start];
        bool first = nc > 0;  // an internal node whose children are all leaves (uniform per block)
        for (int k = 0; k < nc; ++k) first = first && t.node_nchild[t.node_first_child[start] + k] == 0;
        if (!first) continue;
        for (int node = start;;) {
            m2m_node(node);
            __threadfence();  // this thread's writes of node's data before the counter moves
            __syncthreads();
            const int parent = t.node_parent[node];
            if (parent < 0) break;  // uniform: the root
            if (threadIdx.x == 0) {
                climb = atomicSub(pending + parent, 1) == 1;  // the parent's last internal child
                __threadfence();
            }
            __syncthreads();
            if (!climb) break;
            node = parent;
        }
    }
}

// Far-field coefficients B^{0..3}_{m,k} of every node in canonical (order-pm Horner) layout.
__global__ void coeff_kernel(Octree t, int pm, const int4* __restrict__ ent, int n_ent,
                             const double* __restrict__ node_mom, double4* __restrict__ B64,
                             float4* __restrict__ B32, int heavy_cap) {
    const int nn = min(t.counters[1], heavy_cap);
    const int nm = mono_count(pm);
    for (int node = blockIdx.x; node < nn; node += gridDim.x) {
        const double* mom = node_mom + (size_t)node * nm;
        for (int i = threadIdx.x; i < n_ent; i += blockDim.x) {
            const int4 mk = ent[i];  // (m, a, b, c)
            const int m = mk.x, a = mk.y, b = mk.z, c = mk.w, q = a + b + c;
            double n0 = 0, n1 = 0, n2 = 0, n3 = 0;
            for (int j0 = 0; j0 <= m; ++j0) {
                for (int j1 = 0; j1 <= m - j0; ++j1) {
                    const int j2 = m - j0 - j1;
                    const double mult = c_fact[m] / (c_fact[j0] * c_fact[j1] * c_fact[j2]);
                    const int A = a + 2 * j0, Bb = b + 2 * j1, Cc = c + 2 * j2;
                    n0 += mult * mom[mono_index(A, Bb, Cc, pm)];
                    n1 += mult * mom[mono_index(A + 1, Bb, Cc, pm)];
                    n2 += mult * mom[mono_index(A, Bb + 1, Cc, pm)];
                    n3 += mult * mom[mono_index(A, Bb, Cc + 1, pm)];
                }
            }
            const double pre = ((m & 1) ? -1.0 : 1.0) * c_binom[q + m][m] * ((q & 1) ? -1.0 : 1.0) *
                               (double)(1ull << q) * c_fact[q] / (c_fact[a] * c_fact[b] * c_fact[c]);
            const double4 v = make_double4(pre * n0, pre * n1, pre * n2, pre * n3);
            B64[(size_t)node * n_ent + i] = v;
            B32[(size_t)node * n_ent + i] = make_float4((float)v.x, (float)v.y, (float)v.z, (float)v.w);
        }
    }
}

// Scalar far-field coefficients of the 1/|x - y| kernel (Gegenbauer index 1/2), order-pm Horner layout,
// rows padded to `stride` entries.  With d = c - x, e = d/|d|^2, s = 1/|d|^2 and r = y - c:
//   sum_j w_j / |x - y_j| = (1/|d|) sum_{m,k} A_{m,k} e^k s^m,
//   A_{m,k} = (-1)^(m+|k|) g(|k|+m) 2^|k| / k! sum_{|j|=m} M_{k+2j} / j!,  g(n) = Gamma(n+1/2)/Gamma(1/2),
// from the generating function 1/sqrt(1 - 2 t u + u^2) = sum_n C_n^(1/2)(t) u^n.
__global__ void coeff_scalar_kernel(Octree t, int pm, const int4* __restrict__ ent, int n_ent, int stride,
                                    const double* __restrict__ node_mom, double* __restrict__ A64,
                                    float* __restrict__ A32, int heavy_cap) {
    const int nn = min(t.counters[1], heavy_cap);
    const int nm = mono_count(pm);
    for (int node = blockIdx.x; node < nn; node += gridDim.x) {
        const double* mom = node_mom + (size_t)node * nm;
        for (int i = threadIdx.x; i < stride; i += blockDim.x) {
            double v = 0.0;
            if (i < n_ent) {
                const int4 mk = ent[i];  // (m, a, b, c)
                const int m = mk.x, a = mk.y, b = mk.z, c = mk.w, q = a + b + c;
                double n0 = 0;
                for (int j0 = 0; j0 <= m; ++j0)
                    for (int j1 = 0; j1 <= m - j0; ++j1) {
                        const int j2 = m - j0 - j1;
                        n0 += mom[mono_index(a + 2 * j0, b + 2 * j1, c + 2 * j2, pm)] /
                              (c_fact[j0] * c_fact[j1] * c_fact[j2]);
                    }
                double g = 1.0;  // Gamma(q+m+1/2) / Gamma(1/2)
                for (int k = 0; k < q + m; ++k) g *= (double)k + 0.5;
                v = (((m + q) & 1) ? -1.0 : 1.0) * g * (double)(1ull << q) / (c_fact[a] * c_fact[b] * c_fact[c]) * n0;
            }
            A64[(size_t)node * stride + i] = v;
            A32[(size_t)node * stride + i] = (float)v;
        }
    }
}

// Target batches.  Targets sorted by Morton key are cut into batches of at most kBatch consecutive
// targets that also share one octree cell of level `level` (cells of edge 2/2^level): consecutive
// Morton positions can be far apart across a cell boundary, and a batch's radius decides how many
// clusters it can accept.  bflag[q] = 1 where a batch starts: one thread per target finds the first
// target of its cell by binary search in the sorted keys (batches start every kBatch targets from there).
__global__ void batch_flags_kernel(const uint64_t* __restrict__ keys, int64_t n, int shift, int32_t* __restrict__ bflag) {
    for (int64_t q = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; q < n; q += (int64_t)gridDim.x * blockDim.x) {
        const uint64_t cell = keys[q] >> shift;
        int64_t lo = 0, hi = q;  // smallest j <= q in the same cell
        while (lo < hi) {
            const int64_t mid = (lo + hi) >> 1;
            if ((keys[mid] >> shift) < cell) lo = mid + 1;
            else hi = mid;
        }
        bflag[q] = ((q - lo) % kBatch) == 0;
    }
}

// batch_first[b] = first sorted target of batch b (b < n_batches), batch_first[n_batches] = n; the number
// of batches goes to *nbat.  bscan is the exclusive scan of bflag over n + 1 entries.
__global__ void batch_first_kernel(const int32_t* __restrict__ bscan, int64_t n, int32_t* __restrict__ batch_first,
                                   int32_t* __restrict__ nbat, int64_t cap) {
    for (int64_t q = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; q <= n; q += (int64_t)gridDim.x * blockDim.x) {
        const int32_t b = bscan[q];
        const bool start = q == n || bscan[q + 1] != b;
        if (start && b <= cap) batch_first[b] = (int32_t)q;
        if (q == n) *nbat = b;
    }
}

// Per batch: gather its targets into tgt_sorted, centre (mean) and radius.
__global__ void __launch_bounds__(kBatch) batch_kernel(const double4* __restrict__ X, const int32_t* __restrict__ tperm,
                                                       const int32_t* __restrict__ batch_first,
                                                       const int32_t* __restrict__ nbat, double4* __restrict__ tgt_sorted,
                                                       double4* __restrict__ batch_ctr) {
    __shared__ double sh[32];
    if ((int)blockIdx.x >= *nbat) return;  // uniform per block
    const int64_t q0 = batch_first[blockIdx.x], q1 = batch_first[blockIdx.x + 1];
    const int64_t q = q0 + threadIdx.x;
    double4 p = make_double4(0, 0, 0, 0);
    const bool ok = q < q1;
    if (ok) {
        p = X[tperm[q]];
        tgt_sorted[q] = p;
    }
    const int cnt = (int)(q1 - q0);
    const double cx = block_sum(ok ? p.x : 0.0, sh) / cnt, cy = block_sum(ok ? p.y : 0.0, sh) / cnt,
                 cz = block_sum(ok ? p.z : 0.0, sh) / cnt;
    double r = 0;
    if (ok) r = sqrt((p.x - cx) * (p.x - cx) + (p.y - cy) * (p.y - cy) + (p.z - cz) * (p.z - cz));
    r = block_max(r, sh);
    if (threadIdx.x == 0) batch_ctr[blockIdx.x] = make_double4(cx, cy, cz, r);
}

struct TraverseArgs {
    Octree t;
    const double4* node_ctr;
    const double4* batch_ctr;
    const int32_t* batch_first;
    const int32_t* nbat;
    int64_t n_batches;  // capacity (launch size); *nbat batches exist
    double theta;
    int order;
    int direct_below;
    int fill;  // 0 = count, 1 = fill
    int32_t* far_cnt;  // far lists are bucketed by order: row P (stride nb1) holds every batch's order-P entries
    int32_t* near_cnt;
    const int32_t* far_off;
    const int32_t* near_off;
    int2* far_list;
    int2* near_list;
    int64_t far_cap, near_cap;
    int64_t nb1;  // row stride of far_cnt / far_off (n_batches + 1)
    int32_t* flags;
    unsigned long long* pair_counts;  // [0] target-cluster far evaluations, [1] target-source near pairs,
                                      // [2] far coefficient evaluations (sum over far evaluations of E(P))
    // learned order selection (learned != 0): the MLP picks each accepted pair's order
    int learned;
    int max_order;
    int order_bias;  // added to every order the selector picks (capped at max_order)
    double eps;
    CutoffTable ct;
    const float* node_feat;
    const double* node_wabs;
    const __nv_bfloat16* mlp_w;
    const float* mlp_norm;
    uint8_t* decisions;  // n_batches x kDecisionCap selector classes (count pass writes, fill pass reads)
    int heavy_cap;       // nodes with moments / coefficients: only these can be far clusters
    uint32_t* near_work;  // count pass: each batch's near-field (target, source) pairs, saturated at 2^32 - 1
    uint32_t* far_work;   // count pass: each batch's far coefficient evaluations, saturated at 2^32 - 1
};

constexpr int kWarpStack = 1024;
constexpr int kDecisionCap = 1024;  // cached selector decisions per batch

// ---------------------------------------------------------------------------------- learned order
// Per node: log10 radius, log10 sum|w|, log10 of the Frobenius norms of the degree-2/4/6 moment tensors
// about the centre, log10 count, level (8th slot unused).
__global__ void node_feature_kernel(Octree t, int pm, const double4* __restrict__ node_ctr,
                                    const double* __restrict__ node_wabs, const double* __restrict__ node_mom,
                                    float* __restrict__ node_feat, int heavy_cap) {
    const int nn = min(t.counters[1], heavy_cap);
    const int nm = mono_count(pm);
    for (int node = blockIdx.x * blockDim.x + threadIdx.x; node < nn; node += gridDim.x * blockDim.x) {
        const double* mom = node_mom + (size_t)node * nm;
        double norm[3] = {0, 0, 0};
        for (int d = 0; d < 3; ++d) {
            const int n = 2 * (d + 1);
            if (n > pm) continue;
            for (int a = 0; a <= n; ++a)
                for (int b = 0; a + b <= n; ++b) {
                    const double v = mom[mono_index(a, b, n - a - b, pm)];
                    norm[d] += v * v;
                }
        }
        float* f = node_feat + (size_t)node * kMlpIn;
        f[0] = (float)log10(fmax(node_ctr[node].w, 1e-30));
        f[1] = (float)log10(fmax(node_wabs[node], 1e-30));
        for (int d = 0; d < 3; ++d) f[2 + d] = (float)log10(fmax(sqrt(norm[d]), 1e-30));
        f[5] = (float)log10((double)max(t.node_end[node] - t.node_start[node], 1));
        f[6] = (float)t.node_level[node];
        f[7] = 0.0f;
    }
}

// The 8 MLP inputs of a (batch, cluster) pair.  With R' = |x_batch - c| - r_batch the distance from the
// centre to the closest point of the batch's ball and tau = eps * sum|w|_all the per-pair error budget
// (in units of |mult|), the moment features are log10(2 |M_n| / (R'^(n+1) tau)) -- the size of the
// degree-n term of the expansion relative to the budget -- and the monopole-like feature is
// log10(2 sum|w|_c / (R' tau)).
__device__ __forceinline__ void pair_features(const double4& bc, const double4& c, const float* nf, float log_s,
                                              float* f) {
    const double dx = bc.x - c.x, dy = bc.y - c.y, dz = bc.z - c.z;
    const double Rp = fmax(sqrt(dx * dx + dy * dy + dz * dz) - bc.w, 1e-12);
    const float lr = (float)log10(Rp);
    f[0] = nf[0];
    f[1] = nf[0] - lr;
    f[2] = nf[2] + log_s - 3.0f * lr;
    f[3] = nf[3] + log_s - 5.0f * lr;
    f[4] = nf[4] + log_s - 7.0f * lr;
    f[5] = nf[5];
    f[6] = nf[6];
    f[7] = nf[1] + log_s - lr;
}

// log10(2 / tau), tau = eps * sum|w| over all sources (the root's sum)
__device__ __forceinline__ float log_budget(const double* node_wabs, double eps) {
    return (float)log10(2.0 / fmax(eps * node_wabs[0], 1e-300));
}

// One warp per target batch walks the source tree breadth-first, up to 32 nodes per step: (batch, node)
// pairs that pass the acceptance test go to the far list with the order to use; leaves that fail it,
// and accepted clusters too small to be worth an expansion, go to the near list as leaf-id ranges.
// Entries are appended in lane order, so the lists are deterministic.
// Registers capped for 4 resident blocks per SM (16 warps): the count pass, which runs the selector MLP,
// is latency-bound, and at its natural 140 registers only 3 blocks fit (measured 1.52 -> 1.43 ms at icos L8).
#ifndef LPM_TRAVERSE_MIN_BLOCKS
#define LPM_TRAVERSE_MIN_BLOCKS 4
#endif
__global__ void __launch_bounds__(128, LPM_TRAVERSE_MIN_BLOCKS) traverse_kernel(TraverseArgs A) {
    __shared__ int sstack[4][kWarpStack];
    __shared__ int pcnt[4][kPMax + 1];  // per warp: far entries of each order so far
    __shared__ __align__(16) __nv_bfloat16 mw[kMlpParams];
    __shared__ __align__(16) __nv_bfloat16 mxs[4][32 * 16];  // per warp: the selector's input rows
    __shared__ float mnorm[2 * kMlpIn];
    if (A.learned) {  // uniform per launch
        for (int i = threadIdx.x; i < kMlpParams; i += blockDim.x) mw[i] = A.mlp_w[i];
        for (int i = threadIdx.x; i < 2 * kMlpIn; i += blockDim.x) mnorm[i] = A.mlp_norm[i];
        __syncthreads();
    }
    const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int64_t b = (int64_t)blockIdx.x * 4 + w;
    if (A.fill && b == 0 && lane == 0 && A.t.counters[1] > A.heavy_cap) atomicOr(&A.flags[0], 16);
    if (b >= A.n_batches) return;  // uniform per warp
    const Octree& t = A.t;
    const unsigned full = 0xffffffffu, lt = (1u << lane) - 1u;
    int* st = sstack[w];
    if (lane <= kPMax) pcnt[w][lane] = 0;
    if (t.counters[1] == 0 || t.counters[0] == 0 || b >= *A.nbat) {
        if (!A.fill) {
            if (lane <= kPMax) A.far_cnt[lane * A.nb1 + b] = 0;
            if (lane == 0) {
                A.near_cnt[b] = 0;
                A.near_work[b] = 0;
                A.far_work[b] = 0;
            }
        }
        return;
    }
    const double4 bc = A.batch_ctr[b];
    const unsigned long long nb = (unsigned long long)(A.batch_first[b + 1] - A.batch_first[b]);
    const float log_s = A.learned ? log_budget(A.node_wabs, A.eps) : 0.0f;
    int size = 1;
    if (lane == 0) st[0] = 0;
    __syncwarp();
    int nnear = 0, ndec = 0;
    unsigned long long far_pairs = 0, near_pairs = 0, far_terms = 0;
    const int64_t noff = A.fill ? A.near_off[b] : 0;
    while (size > 0) {
        const int m = min(32, size);
        const int node = lane < m ? st[size - 1 - lane] : -1;
        __syncwarp();
        size -= m;
        int kind = 0, nch = 0, lo = 0, hi = 0, cnt = 0, fc = 0, P = A.order;
        double4 c = make_double4(0, 0, 0, 0);
        int s = 0, e = 0, nc = 0;
        bool far_ok = false;
        if (node >= 0) {
            c = A.node_ctr[node];
            s = t.node_start[node];
            e = t.node_end[node];
            const double dx = bc.x - c.x, dy = bc.y - c.y, dz = bc.z - c.z;
            const double R = sqrt(dx * dx + dy * dy + dz * dz);
            far_ok = R > bc.w && c.w < A.theta * (R - bc.w) && node < A.heavy_cap;
            nc = t.node_nchild[node];
        }
        int cut = A.direct_below;
        if (A.learned) {  // uniform per launch
            // the selector's order; "no order meets the budget" opens a cluster large enough to be worth
            // opening and sums a leaf or a small cluster directly.  The count pass caches each batch's
            // first kDecisionCap decisions (in visiting order) for the fill pass.
            const unsigned okm = __ballot_sync(full, far_ok);
            const int idx = ndec + __popc(okm & lt);
            ndec += __popc(okm);
            uint8_t* dec = A.decisions + (size_t)b * kDecisionCap;
            int cls = -1;
            if (far_ok && A.fill && idx < kDecisionCap) cls = dec[idx];
            const bool need = far_ok && cls < 0;
            if (__any_sync(full, need)) {  // the whole warp runs the selector on the tensor cores
                float f[kMlpIn];
#pragma unroll
                for (int i = 0; i < kMlpIn; ++i) f[i] = mnorm[i];  // finite filler for lanes without a pair
                if (need) pair_features(bc, c, A.node_feat + (size_t)node * kMlpIn, log_s, f);
                const int c2 = mlp_warp_argmax(mw, mnorm, f, mxs[w]);
                if (need) {
                    cls = c2;
                    if (!A.fill && idx < kDecisionCap) dec[idx] = (uint8_t)cls;
                }
            }
            if (far_ok) {
                P = cls == kMlpDirectClass ? 0 : min(cls + 1 + A.order_bias, A.max_order);
                cut = P > 0 ? A.ct.direct_below[P] : 0x7fffffff;
                if (P == 0 && nc > 0 && e - s >= A.ct.direct_below[A.max_order]) far_ok = false;
            }
        }
        if (node >= 0) {
            if (far_ok && e - s >= cut) {
                kind = 1;
            } else if (far_ok || nc == 0) {
                kind = 2;
                lo = t.leaf_flag[s];
                hi = t.leaf_flag[e] - 1;
                cnt = e - s;
            } else {
                kind = 3;
                nch = nc;
                fc = t.node_first_child[node];
            }
        }
        const unsigned fm = __ballot_sync(full, kind == 1);
        if (fm) {  // warp-uniform: rank each far entry among this step's entries of its order, in lane order
            const unsigned grp = __match_any_sync(full, kind == 1 ? P : 64 + lane);
            const int rank = __popc(grp & lt);
            const int base = kind == 1 ? pcnt[w][P] : 0;
            __syncwarp();
            if (kind == 1) {
                if (rank == 0) pcnt[w][P] = base + __popc(grp);
                if (A.fill) {
                    const int64_t at = A.far_off[P * A.nb1 + b] + base + rank;
                    if (at < A.far_cap) A.far_list[at] = make_int2(node, P);
                    else atomicOr(&A.flags[0], 1);
                }
            }
            __syncwarp();
        }
        far_pairs += (unsigned long long)__popc(fm) * nb;
        const unsigned nm = __ballot_sync(full, kind == 2);
        if (kind == 2 && A.fill) {
            const int64_t at = noff + nnear + __popc(nm & lt);
            if (at < A.near_cap) A.near_list[at] = make_int2(lo, hi);
            else atomicOr(&A.flags[0], 2);
        }
        nnear += __popc(nm);
        unsigned long long np = (unsigned long long)cnt * nb;
        unsigned long long ft = kind == 1 ? (unsigned long long)entries_for(P) * nb : 0ull;
        for (int o = 16; o > 0; o >>= 1) {
            np += __shfl_xor_sync(full, np, o);
            ft += __shfl_xor_sync(full, ft, o);
        }
        near_pairs += np;
        far_terms += ft;
        // push the children of split nodes
        int incl = nch;
        for (int o = 1; o < 32; o <<= 1) {
            const int v = __shfl_up_sync(full, incl, o);
            if (lane >= o) incl += v;
        }
        const int total = __shfl_sync(full, incl, 31);
        if (size + total > kWarpStack) {
            if (lane == 0) atomicOr(&A.flags[0], 4);
        } else if (kind == 3) {
            const int base = size + incl - nch;
            for (int k = 0; k < nch; ++k) st[base + k] = fc + nch - 1 - k;
        }
        __syncwarp();
        if (size + total <= kWarpStack) size += total;
    }
    if (!A.fill && lane <= kPMax) A.far_cnt[lane * A.nb1 + b] = pcnt[w][lane];
    if (!A.fill && lane == 0) {
        A.near_cnt[b] = nnear;
        A.near_work[b] = (uint32_t)min(near_pairs, 0xffffffffull);
        A.far_work[b] = (uint32_t)min(far_terms, 0xffffffffull);
        atomicAdd(&A.pair_counts[0], far_pairs);
        atomicAdd(&A.pair_counts[1], near_pairs);
        atomicAdd(&A.pair_counts[2], far_terms);
    }
}

// ---------------------------------------------------------------------------------- batch schedule
// Batches in decreasing order of work, bucketed by log2(work) in half-octave steps: a persistent kernel
// that takes batches in this order from an atomic ticket ends on its smallest batches, so few SMs idle at
// its tail.  Each batch is still computed by one block, so the results do not depend on the order.
constexpr int kSchedBuckets = 64;
// the solver's schedule scratch (int32): near buckets and cursors, far buckets and cursors, then one ticket
// for the near launch and one per far order
constexpr int kAuxNearHist = 0, kAuxNearCur = 64, kAuxFarHist = 128, kAuxFarCur = 192, kAuxNearTicket = 256,
              kAuxFarTicket = 257, kAuxInts = 257 + 16;

__device__ __forceinline__ int sched_bucket(uint32_t work) {
    const int l2 = (int)(2.0f * __log2f((float)work + 1.0f));
    return kSchedBuckets - 1 - min(max(l2, 0), kSchedBuckets - 1);
}

// hist[0:64] and cursor[0:64] zeroed by the caller.
__global__ void sched_hist_kernel(const uint32_t* __restrict__ work, const int32_t* __restrict__ nbat,
                                  int32_t* __restrict__ hist) {
    const int n = *nbat;
    for (int b = blockIdx.x * blockDim.x + threadIdx.x; b < n; b += gridDim.x * blockDim.x)
        atomicAdd(&hist[sched_bucket(work[b])], 1);
}

__global__ void sched_scatter_kernel(const uint32_t* __restrict__ work, const int32_t* __restrict__ nbat,
                                     const int32_t* __restrict__ hist, int32_t* __restrict__ cursor,
                                     int32_t* __restrict__ order) {
    __shared__ int base[kSchedBuckets];
    if (threadIdx.x == 0) {
        int acc = 0;
        for (int k = 0; k < kSchedBuckets; ++k) {
            base[k] = acc;
            acc += hist[k];
        }
    }
    __syncthreads();
    const int n = *nbat;
    for (int b = blockIdx.x * blockDim.x + threadIdx.x; b < n; b += gridDim.x * blockDim.x) {
        const int k = sched_bucket(work[b]);
        order[base[k] + atomicAdd(&cursor[k], 1)] = b;
    }
}

// The next batch of a persistent kernel's block: order[ticket++] while tickets last, else -1.  ticket is
// zeroed before the launch.
__device__ __forceinline__ int next_batch(int32_t* ticket, const int32_t* __restrict__ order, int nbat, int* slot) {
    __syncthreads();  // every thread is done with the previous batch's shared memory
    if (threadIdx.x == 0) {
        const int k = atomicAdd(ticket, 1);
        *slot = k < nbat ? order[k] : -1;
    }
    __syncthreads();
    return *slot;
}

// ---------------------------------------------------------------------------------- far field
template <int P, typename T, typename T4>
__device__ __forceinline__ void horner(const T4* __restrict__ Bc, T e0, T e1, T e2, T s, T& g0, T& g1, T& g2,
                                       T& g3) {
    // Each chain starts from its leading term (an FMA onto a zero accumulator cannot be folded away by
    // the compiler, since 0 * e is not 0 for infinite e): one FMA per coefficient after the first.
    int q = 0;
    T G0 = 0, G1 = 0, G2 = 0, G3 = 0;
#pragma unroll
    for (int m = (P - 1) / 2; m >= 0; --m) {
        const int Q = P - 2 * m;
        T P0 = 0, P1 = 0, P2 = 0, P3 = 0;
#pragma unroll
        for (int a = Q - 1; a >= 0; --a) {
            T Q0 = 0, Q1 = 0, Q2 = 0, Q3 = 0;
#pragma unroll
            for (int b = Q - 1 - a; b >= 0; --b) {
                T R0 = 0, R1 = 0, R2 = 0, R3 = 0;
#pragma unroll
                for (int c = Q - 1 - a - b; c >= 0; --c) {
                    const T4 v = Bc[q++];
                    if (c == Q - 1 - a - b) {
                        R0 = v.x; R1 = v.y; R2 = v.z; R3 = v.w;
                    } else {
                        R0 = fma(R0, e2, v.x); R1 = fma(R1, e2, v.y); R2 = fma(R2, e2, v.z); R3 = fma(R3, e2, v.w);
                    }
                }
                if (b == Q - 1 - a) {
                    Q0 = R0; Q1 = R1; Q2 = R2; Q3 = R3;
                } else {
                    Q0 = fma(Q0, e1, R0); Q1 = fma(Q1, e1, R1); Q2 = fma(Q2, e1, R2); Q3 = fma(Q3, e1, R3);
                }
            }
            if (a == Q - 1) {
                P0 = Q0; P1 = Q1; P2 = Q2; P3 = Q3;
            } else {
                P0 = fma(P0, e0, Q0); P1 = fma(P1, e0, Q1); P2 = fma(P2, e0, Q2); P3 = fma(P3, e0, Q3);
            }
        }
        if (m == (P - 1) / 2) {
            G0 = P0; G1 = P1; G2 = P2; G3 = P3;
        } else {
            G0 = fma(G0, s, P0); G1 = fma(G1, s, P1); G2 = fma(G2, s, P2); G3 = fma(G3, s, P3);
        }
    }
    g0 = G0; g1 = G1; g2 = G2; g3 = G3;
}

// FP32 Horner scheme with the four components in two packed pairs (fma.rn.f32x2, sm_100): half the FMA
// instructions per coefficient for the same lane work and the same rounding (measured: far field 17-19%
// faster).
template <int P>
__device__ __forceinline__ void horner_f32x2(const float4* __restrict__ Bc, float e0, float e1, float e2, float s,
                                             float& g0, float& g1, float& g2, float& g3) {
    int q = 0;
    float G0 = 0, G1 = 0, G2 = 0, G3 = 0;
#pragma unroll
    for (int m = (P - 1) / 2; m >= 0; --m) {
        const int Q = P - 2 * m;
        float P0 = 0, P1 = 0, P2 = 0, P3 = 0;
#pragma unroll
        for (int a = Q - 1; a >= 0; --a) {
            float Q0 = 0, Q1 = 0, Q2 = 0, Q3 = 0;
#pragma unroll
            for (int b = Q - 1 - a; b >= 0; --b) {
                float R0 = 0, R1 = 0, R2 = 0, R3 = 0;
#pragma unroll
                for (int c = Q - 1 - a - b; c >= 0; --c) {
                    const float4 v = Bc[q++];
                    if (c == Q - 1 - a - b) {  // leading term: no FMA (see horner)
                        R0 = v.x; R1 = v.y; R2 = v.z; R3 = v.w;
                    } else {
                        fma2p(R0, R1, R0, R1, e2, v.x, v.y);
                        fma2p(R2, R3, R2, R3, e2, v.z, v.w);
                    }
                }
                if (b == Q - 1 - a) {
                    Q0 = R0; Q1 = R1; Q2 = R2; Q3 = R3;
                } else {
                    fma2p(Q0, Q1, Q0, Q1, e1, R0, R1);
                    fma2p(Q2, Q3, Q2, Q3, e1, R2, R3);
                }
            }
            if (a == Q - 1) {
                P0 = Q0; P1 = Q1; P2 = Q2; P3 = Q3;
            } else {
                fma2p(P0, P1, P0, P1, e0, Q0, Q1);
                fma2p(P2, P3, P2, P3, e0, Q2, Q3);
            }
        }
        if (m == (P - 1) / 2) {
            G0 = P0; G1 = P1; G2 = P2; G3 = P3;
        } else {
            fma2p(G0, G1, G0, G1, s, P0, P1);
            fma2p(G2, G3, G2, G3, s, P2, P3);
        }
    }
    g0 = G0; g1 = G1; g2 = G2; g3 = G3;
}

// Adds 2 [(x cross d) G0 + x cross G] of one cluster to V, d = c - x.
template <int P, typename T, typename T4>
__device__ __forceinline__ void far_one(const T4* Bc, const double4& x, const double4& c, double* V) {
    const double dx = c.x - x.x, dy = c.y - x.y, dz = c.z - x.z;
    const double r2 = dx * dx + dy * dy + dz * dz;
    const double inv = 1.0 / r2;
    T g0, g1, g2, g3;
    horner<P, T, T4>(Bc, (T)(dx * inv), (T)(dy * inv), (T)(dz * inv), (T)inv, g0, g1, g2, g3);
    const double G0 = 2.0 * inv * (double)g0, Gx = 2.0 * inv * (double)g1, Gy = 2.0 * inv * (double)g2,
                 Gz = 2.0 * inv * (double)g3;
    V[0] += (x.y * dz - x.z * dy) * G0 + (x.y * Gz - x.z * Gy);
    V[1] += (x.z * dx - x.x * dz) * G0 + (x.z * Gx - x.x * Gz);
    V[2] += (x.x * dy - x.y * dx) * G0 + (x.x * Gy - x.y * Gx);
}

template <typename T, typename T4>
__device__ void far_dispatch(int P, const T4* Bc, const double4& x, const double4& c, double* V) {
    switch (P) {
        case 1: far_one<1, T, T4>(Bc, x, c, V); break;
        case 2: far_one<2, T, T4>(Bc, x, c, V); break;
        case 3: far_one<3, T, T4>(Bc, x, c, V); break;
        case 4: far_one<4, T, T4>(Bc, x, c, V); break;
        case 5: far_one<5, T, T4>(Bc, x, c, V); break;
        case 6: far_one<6, T, T4>(Bc, x, c, V); break;
        case 7: far_one<7, T, T4>(Bc, x, c, V); break;
        case 8: far_one<8, T, T4>(Bc, x, c, V); break;
        case 9: far_one<9, T, T4>(Bc, x, c, V); break;
        case 10: far_one<10, T, T4>(Bc, x, c, V); break;
        case 11: far_one<11, T, T4>(Bc, x, c, V); break;
        case 12: far_one<12, T, T4>(Bc, x, c, V); break;
        default: break;
    }
}

constexpr int kF64From = 8;  // default: orders >= this evaluate in FP64

__device__ __forceinline__ void cp_async16(void* smem, const void* gmem) {
    const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(s), "l"(gmem));
}

__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait_prev() { asm volatile("cp.async.wait_group 1;\n" ::: "memory"); }

template <typename F, typename F4>
__device__ __forceinline__ void fma4(F (&r)[4], F e, const F4& v) {
    r[0] = fma(r[0], e, v.x);
    r[1] = fma(r[1], e, v.y);
    r[2] = fma(r[2], e, v.z);
    r[3] = fma(r[3], e, v.w);
}
template <typename F>
__device__ __forceinline__ void fma4(F (&r)[4], F e, const F (&v)[4]) {
    r[0] = fma(r[0], e, v[0]);
    r[1] = fma(r[1], e, v[1]);
    r[2] = fma(r[2], e, v[2]);
    r[3] = fma(r[3], e, v[3]);
}

// One far entry at one target in F arithmetic.  The cluster's contribution 2 x cross (d g0 + g) / |d|^2
// (d = c - x, g from the order-P Horner scheme, fully unrolled for P) is linear in the target position x, so
// acc sums h = (d g0 + g) / |d|^2 and the caller applies 2 x cross acc once per target.
template <int P, typename F, typename F4>
__device__ __forceinline__ void far_one_acc(const F4* __restrict__ Bc, const double4& x, double cx, double cy,
                                            double cz, double (&acc)[3]) {
    const F dx = (F)(cx - x.x), dy = (F)(cy - x.y), dz = (F)(cz - x.z);
    const F inv = F(1) / (dx * dx + dy * dy + dz * dz);
    F g0, g1, g2, g3;
    if constexpr (sizeof(F) == 4)
        horner_f32x2<P>((const float4*)Bc, dx * inv, dy * inv, dz * inv, inv, g0, g1, g2, g3);
    else
        horner<P, F, F4>(Bc, dx * inv, dy * inv, dz * inv, inv, g0, g1, g2, g3);
    acc[0] += (double)(inv * fma(dx, g0, g1));
    acc[1] += (double)(inv * fma(dy, g0, g2));
    acc[2] += (double)(inv * fma(dz, g0, g3));
}

struct FarArgs {
    const double4* tgt_sorted;
    int64_t n_tgt;
    const int32_t* batch_first;
    const int32_t* nbat;
    const int32_t* far_off;  // row P of the bucketed offsets / counts
    const int32_t* far_cnt;
    const int2* far_list;
    int64_t far_cap;
    const double4* node_ctr;
    const double4* B64;
    const float4* B32;
    int n_ent;
    const int32_t* gtab;  // order-P gather table: canonical index of each Horner-sequence entry
    double* V;
    const int32_t* order;  // batches by decreasing far work (the persistent grid's visiting order)
    int32_t* ticket;       // this launch's ticket, zeroed before it
};

#ifndef LPM_FAR_STAGE_UNITS
#define LPM_FAR_STAGE_UNITS 1024
#endif
#ifndef LPM_FAR_MIN_BLOCKS
#define LPM_FAR_MIN_BLOCKS 6
#endif
constexpr int kFarStageUnits = LPM_FAR_STAGE_UNITS;  // 16-byte units gathered per stage (at least one entry)
constexpr int kFarMinBlocks = LPM_FAR_MIN_BLOCKS;    // resident blocks per SM the far kernels are built for

template <int P, typename F4, int U = kFarStageUnits, int PART = 0>
struct FarShape {
    static constexpr int kUnits = part_entries(P, PART) * (int)(sizeof(F4) / 16);  // per entry
    static constexpr int kK = kUnits >= U ? 1 : (U / kUnits > 32 ? 32 : U / kUnits);
    static constexpr int kStage = kK * kUnits;  // units per stage buffer
    static constexpr size_t kSmem = 2 * (size_t)kStage * 16 + 2 * (size_t)kK * sizeof(double4);
};

// Issue the copies of entries [s0, s0 + n) of the batch's order-P list into one stage: coefficients by
// cp.async, cluster centres by plain stores.
template <int P, typename F4, int NT = kBatch>
__device__ __forceinline__ void far_stage_gather(const FarArgs& A, int64_t s0, int n, float4* buf, double4* ctr) {
    constexpr int kUnits = FarShape<P, F4>::kUnits;
    constexpr int kSub = (int)(sizeof(F4) / 16);
    const F4* base = (const F4*)(kSub == 2 ? (const void*)A.B64 : (const void*)A.B32);
    for (int i = threadIdx.x; i < n * kUnits; i += NT) {
        const int e = i / kUnits, j = i - e * kUnits;
        const int node = A.far_list[s0 + e].x;
        const char* src = (const char*)(base + (size_t)node * A.n_ent + A.gtab[j / kSub]) + 16 * (j % kSub);
        cp_async16(buf + i, src);
    }
    if ((int)threadIdx.x < n) ctr[threadIdx.x] = A.node_ctr[A.far_list[s0 + threadIdx.x].x];
}

// Far field for the order-P bucket: one block per target batch, one thread per target, the order's
// fully unrolled Horner scheme in F arithmetic.  Entries are gathered kK at a time into one half of a
// double buffer (cp.async) while the other half is evaluated; one launch per order keeps every warp of
// the GPU in the same compact code.  Adds to V (cleared before the first order's launch).
template <int P, typename F, typename F4>
__global__ void __launch_bounds__(kBatch, kFarMinBlocks) far_order_kernel(FarArgs A) {
    using S = FarShape<P, F4>;
    extern __shared__ float4 fbuf[];  // 2 stages of S::kStage units, then 2 x kK centres
    double4* ctr = (double4*)(fbuf + 2 * S::kStage);
    __shared__ int slot;
    const int nbat = *A.nbat;
    for (int64_t b = next_batch(A.ticket, A.order, nbat, &slot); b >= 0; b = next_batch(A.ticket, A.order, nbat, &slot)) {
    const int64_t f0 = A.far_off[b], f1 = min(f0 + (int64_t)A.far_cnt[b], A.far_cap);
    if (f0 >= f1) continue;  // uniform per block
    const int64_t q0 = A.batch_first[b], qe = A.batch_first[b + 1];
    const int64_t q = q0 + threadIdx.x;
    const bool live = q0 + (int64_t)(threadIdx.x & ~31) < qe;  // warp-uniform
    const double4 x = q < qe ? A.tgt_sorted[q] : make_double4(0, 0, 1, 0);
    double acc[3] = {0, 0, 0};
    far_stage_gather<P, F4>(A, f0, (int)min((int64_t)S::kK, f1 - f0), fbuf, ctr);
    cp_async_commit();
    int s = 0;
    for (int64_t s0 = f0;; s ^= 1) {
        const int n = (int)min((int64_t)S::kK, f1 - s0);
        const int64_t s1 = s0 + n;
        if (s1 < f1)
            far_stage_gather<P, F4>(A, s1, (int)min((int64_t)S::kK, f1 - s1), fbuf + (size_t)(s ^ 1) * S::kStage,
                                    ctr + (s ^ 1) * S::kK);
        cp_async_commit();
        cp_async_wait_prev();
        __syncthreads();  // stage s resident
        if (live) {
            const F4* Bc = (const F4*)(fbuf + (size_t)s * S::kStage);
            const double4* cs = ctr + s * S::kK;
            for (int k = 0; k < n; ++k)
                far_one_acc<P, F, F4>(Bc + (size_t)k * entries_for(P), x, cs[k].x, cs[k].y, cs[k].z, acc);
        }
        if (s1 >= f1) break;
        __syncthreads();  // stage s consumed before it is refilled
        s0 = s1;
    }
    if (q < qe) {  // V += 2 x cross acc
        const double hx = 2.0 * acc[0], hy = 2.0 * acc[1], hz = 2.0 * acc[2];
        A.V[q] += x.y * hz - x.z * hy;
        A.V[A.n_tgt + q] += x.z * hx - x.x * hz;
        A.V[2 * A.n_tgt + q] += x.x * hy - x.y * hx;
    }
    }
}

// ---- two targets per thread (FP32)
// The Horner scheme of horner_f32x2 for two targets at once: every coefficient read from shared memory
// feeds both targets' chains (four packed FMAs per load instead of two) and each thread carries two
// independent dependency chains.  e[t] = (e0, e1, e2, s) of target t; same arithmetic per target as
// horner_f32x2.
template <int P, int PART = 0>
__device__ __forceinline__ void horner2_f32x2(const float4* __restrict__ Bc, const float (&e)[2][4],
                                              float (&g)[2][4]) {
    int q = 0;
    float G[2][4] = {{0, 0, 0, 0}, {0, 0, 0, 0}};
#pragma unroll
    for (int m = PART == 2 ? 0 : (P - 1) / 2; m >= (PART == 1 ? 1 : 0); --m) {
        const int Q = P - 2 * m;
        float Pa[2][4] = {{0, 0, 0, 0}, {0, 0, 0, 0}};
#pragma unroll
        for (int a = Q - 1; a >= 0; --a) {
            float Qa[2][4] = {{0, 0, 0, 0}, {0, 0, 0, 0}};
#pragma unroll
            for (int b = Q - 1 - a; b >= 0; --b) {
                float R[2][4] = {{0, 0, 0, 0}, {0, 0, 0, 0}};
#pragma unroll
                for (int c = Q - 1 - a - b; c >= 0; --c) {
                    const float4 v = Bc[q++];
#pragma unroll
                    for (int t = 0; t < 2; ++t) {
                        if (c == Q - 1 - a - b) {  // leading term: no FMA (see horner)
                            R[t][0] = v.x; R[t][1] = v.y; R[t][2] = v.z; R[t][3] = v.w;
                        } else {
                            fma2p(R[t][0], R[t][1], R[t][0], R[t][1], e[t][2], v.x, v.y);
                            fma2p(R[t][2], R[t][3], R[t][2], R[t][3], e[t][2], v.z, v.w);
                        }
                    }
                }
#pragma unroll
                for (int t = 0; t < 2; ++t) {
                    if (b == Q - 1 - a) {
                        Qa[t][0] = R[t][0]; Qa[t][1] = R[t][1]; Qa[t][2] = R[t][2]; Qa[t][3] = R[t][3];
                    } else {
                        fma2p(Qa[t][0], Qa[t][1], Qa[t][0], Qa[t][1], e[t][1], R[t][0], R[t][1]);
                        fma2p(Qa[t][2], Qa[t][3], Qa[t][2], Qa[t][3], e[t][1], R[t][2], R[t][3]);
                    }
                }
            }
#pragma unroll
            for (int t = 0; t < 2; ++t) {
                if (a == Q - 1) {
                    Pa[t][0] = Qa[t][0]; Pa[t][1] = Qa[t][1]; Pa[t][2] = Qa[t][2]; Pa[t][3] = Qa[t][3];
                } else {
                    fma2p(Pa[t][0], Pa[t][1], Pa[t][0], Pa[t][1], e[t][0], Qa[t][0], Qa[t][1]);
                    fma2p(Pa[t][2], Pa[t][3], Pa[t][2], Pa[t][3], e[t][0], Qa[t][2], Qa[t][3]);
                }
            }
        }
#pragma unroll
        for (int t = 0; t < 2; ++t) {
            if (m == (PART == 2 ? 0 : (P - 1) / 2)) {
                G[t][0] = Pa[t][0]; G[t][1] = Pa[t][1]; G[t][2] = Pa[t][2]; G[t][3] = Pa[t][3];
            } else {
                fma2p(G[t][0], G[t][1], G[t][0], G[t][1], e[t][3], Pa[t][0], Pa[t][1]);
                fma2p(G[t][2], G[t][3], G[t][2], G[t][3], e[t][3], Pa[t][2], Pa[t][3]);
            }
        }
    }
    if constexpr (PART == 1) {  // the blocks m >= 1 carry one more factor s
#pragma unroll
        for (int c = 0; c < 4; ++c) fma2v(G[0][c], G[1][c], G[0][c], G[1][c], e[0][3], e[1][3], -0.0f, -0.0f);
    }
#pragma unroll
    for (int t = 0; t < 2; ++t)
#pragma unroll
        for (int c = 0; c < 4; ++c) g[t][c] = G[t][c];
}

#ifndef LPM_FAR2_MAX_ORDER
#define LPM_FAR2_MAX_ORDER 11
#endif
#ifndef LPM_FAR2_STAGE_UNITS
#define LPM_FAR2_STAGE_UNITS 768
#endif
#ifndef LPM_FAR2_MIN_BLOCKS
#define LPM_FAR2_MIN_BLOCKS 7
#endif
constexpr int kFar2MaxOrder = LPM_FAR2_MAX_ORDER;  // FP32 orders up to this run two targets per thread (all used)
constexpr int kFar2Threads = kBatch / 2;
constexpr int kFar2StageUnits = LPM_FAR2_STAGE_UNITS;
constexpr int kFar2MinBlocks = LPM_FAR2_MIN_BLOCKS;

// The far2 kernel's per-entry work in FP32 throughout: centres and targets are offsets from a point of the
// batch (its first target), so d = c - x is one FP32 subtraction; 1/|d|^2 by the approximate reciprocal
// (1 ulp).  A cluster adds x cross (2/|d|^2) (d g0 + g) to the target's sum, linear in the target position x,
// so the kernel sums only h = (1/|d|^2) (d g0 + g) over the clusters and applies 2 x cross (.) once per
// target at the end in FP64: acc32 += h in FP32 over a stage, folded into FP64 once per stage.  Every step
// runs on the two targets together (fma.rn.f32x2, each lane rounding as the scalar operation); xo holds the
// targets' offsets and c the centre's.
template <int P, int PART = 0>
__device__ __forceinline__ void far_one_acc2_f32(const float4* __restrict__ Bc, const float (&xo)[2][3],
                                                 const float4 c, float (&acc32)[2][3]) {
    float d[2][3], e[2][4], g[2][4], r0, r1;
    fma2p(d[0][0], d[1][0], xo[0][0], xo[1][0], -1.0f, c.x, c.x);  // c - xo, one rounding
    fma2p(d[0][1], d[1][1], xo[0][1], xo[1][1], -1.0f, c.y, c.y);
    fma2p(d[0][2], d[1][2], xo[0][2], xo[1][2], -1.0f, c.z, c.z);
    fma2v(r0, r1, d[0][0], d[1][0], d[0][0], d[1][0], -0.0f, -0.0f);
    fma2v(r0, r1, d[0][1], d[1][1], d[0][1], d[1][1], r0, r1);
    fma2v(r0, r1, d[0][2], d[1][2], d[0][2], d[1][2], r0, r1);
    e[0][3] = rcp32(r0);
    e[1][3] = rcp32(r1);
#pragma unroll
    for (int k = 0; k < 3; ++k) fma2v(e[0][k], e[1][k], d[0][k], d[1][k], e[0][3], e[1][3], -0.0f, -0.0f);
    horner2_f32x2<P, PART>(Bc, e, g);
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        float h0, h1;
        fma2v(h0, h1, d[0][k], d[1][k], g[0][0], g[1][0], g[0][k + 1], g[1][k + 1]);
        fma2v(acc32[0][k], acc32[1][k], h0, h1, e[0][3], e[1][3], acc32[0][k], acc32[1][k]);
    }
}

// Stage gather of the far2 kernel: coefficients by cp.async as far_stage_gather, cluster centres as FP32
// offsets from the block's origin o.
template <int P, int PART = 0>
__device__ __forceinline__ void far2_stage_gather(const FarArgs& A, int64_t s0, int n, float4* buf, float4* ctr,
                                                  const double4& o) {
    constexpr int kUnits = FarShape<P, float4, kFarStageUnits, PART>::kUnits;
    for (int i = threadIdx.x; i < n * kUnits; i += kFar2Threads) {
        const int e = i / kUnits, j = i - e * kUnits;
        const int node = A.far_list[s0 + e].x;
        cp_async16(buf + i, A.B32 + (size_t)node * A.n_ent + A.gtab[j]);
    }
    if ((int)threadIdx.x < n) {
        const double4 c = A.node_ctr[A.far_list[s0 + threadIdx.x].x];
        ctr[threadIdx.x] = make_float4((float)(c.x - o.x), (float)(c.y - o.y), (float)(c.z - o.z), 0.0f);
    }
}

// One batch b of the far2 kernel (the whole block); fbuf: 2 stages of S::kStage units, then 2 x kK centres
// (FP32 offsets).
template <int P, int PART = 0>
__device__ __forceinline__ void far2_batch(const FarArgs& A, int64_t b, float4* fbuf) {
    using S = FarShape<P, float4, kFar2StageUnits, PART>;
    float4* ctr = fbuf + 2 * S::kStage;
    const int64_t f0 = A.far_off[b], f1 = min(f0 + (int64_t)A.far_cnt[b], A.far_cap);
    if (f0 >= f1) return;  // uniform per block
    const int64_t q0 = A.batch_first[b], qe = A.batch_first[b + 1];
    // warp w holds targets 64 w .. 64 w + 63 of the batch (lane l: 64 w + l and 64 w + l + 32), so a warp past
    // the batch's last target idles as a whole (batches average ~109 of 128 targets)
    const int64_t qa = q0 + 64 * (threadIdx.x >> 5) + (threadIdx.x & 31), qb = qa + 32;
    const bool live = q0 + 64 * (int64_t)(threadIdx.x >> 5) < qe;  // warp-uniform
    const double4 o = A.tgt_sorted[q0];  // the block's origin for FP32 offsets
    float xo[2][3];
#pragma unroll
    for (int t = 0; t < 2; ++t) {
        const int64_t q = t ? qb : qa;
        const double4 p = q < qe ? A.tgt_sorted[q] : make_double4(0, 0, 1, 0);
        xo[t][0] = (float)(p.x - o.x); xo[t][1] = (float)(p.y - o.y); xo[t][2] = (float)(p.z - o.z);
    }
    double acc[2][3] = {{0, 0, 0}, {0, 0, 0}};
    far2_stage_gather<P, PART>(A, f0, (int)min((int64_t)S::kK, f1 - f0), fbuf, ctr, o);
    cp_async_commit();
    int s = 0;
    for (int64_t s0 = f0;; s ^= 1) {
        const int n = (int)min((int64_t)S::kK, f1 - s0);
        const int64_t s1 = s0 + n;
        if (s1 < f1)
            far2_stage_gather<P, PART>(A, s1, (int)min((int64_t)S::kK, f1 - s1), fbuf + (size_t)(s ^ 1) * S::kStage,
                                 ctr + (s ^ 1) * S::kK, o);
        cp_async_commit();
        cp_async_wait_prev();
        __syncthreads();  // stage s resident
        if (live) {
            const float4* Bc = fbuf + (size_t)s * S::kStage;
            const float4* cs = ctr + s * S::kK;
            float acc32[2][3] = {{0, 0, 0}, {0, 0, 0}};
            for (int k = 0; k < n; ++k)
                far_one_acc2_f32<P, PART>(Bc + (size_t)k * part_entries(P, PART), xo, cs[k], acc32);
#pragma unroll
            for (int t = 0; t < 2; ++t)
#pragma unroll
                for (int c = 0; c < 3; ++c) acc[t][c] += (double)acc32[t][c];
        }
        if (s1 >= f1) break;
        __syncthreads();  // stage s consumed before it is refilled
        s0 = s1;
    }
#pragma unroll
    for (int t = 0; t < 2; ++t) {  // V += 2 x cross (sum of h), x the FP64 target
        const int64_t q = t ? qb : qa;
        if (q >= qe) continue;
        const double4 p = A.tgt_sorted[q];
        const double hx = 2.0 * acc[t][0], hy = 2.0 * acc[t][1], hz = 2.0 * acc[t][2];
        A.V[q] += p.y * hz - p.z * hy;
        A.V[A.n_tgt + q] += p.z * hx - p.x * hz;
        A.V[2 * A.n_tgt + q] += p.x * hy - p.y * hx;
    }
}

// far_order_kernel<P, float, float4> with two targets per thread (targets i and i + 64 of the batch):
// 64 threads per block, stages of kFar2StageUnits, the same double buffering.  Built for 7 blocks per SM
// (128 registers; the odd orders spill up to 128 bytes to L1) with 768-unit stages: measured faster than
// 6 blocks without spills, than more resident blocks with smaller stages (fewer block barriers per
// coefficient) and than fewer blocks with larger ones.
template <int P, int PART = 0>
__global__ void __launch_bounds__(kFar2Threads, kFar2MinBlocks) far_order2_kernel(FarArgs A) {
    extern __shared__ float4 fbuf[];
    __shared__ int slot;
    const int nbat = *A.nbat;
    for (int64_t b = next_batch(A.ticket, A.order, nbat, &slot); b >= 0; b = next_batch(A.ticket, A.order, nbat, &slot))
        far2_batch<P, PART>(A, b, fbuf);
}

// The short orders 1..kFarLowMax of the FP32 far field in one persistent launch: a block takes a batch (in
// decreasing order of its far work) and runs the order-P body for each of these orders in turn, so V receives
// the orders' sums in the order of separate launches (bitwise the same).  As separate launches these orders
// were latency-bound (few clusters per batch, waits on the coefficient gathers), each with its own tail.
constexpr int kFarLowMax = 4;
struct FarLowArgs {
    FarArgs a[kFarLowMax];  // a[P - 1]: order P's arguments; far_cnt null: order P is not in this launch
};

__global__ void __launch_bounds__(kFar2Threads, kFar2MinBlocks) far_low2_kernel(FarLowArgs L,
                                                                               const int32_t* __restrict__ nbat_p,
                                                                               const int32_t* __restrict__ order,
                                                                               int32_t* ticket) {
    static_assert(kFarLowMax == 4 && kFarLowMax < kFarSplitOrder, "orders 1..4, none split");
    extern __shared__ float4 fbuf[];
    __shared__ int slot;
    const int nbat = *nbat_p;
    for (int64_t b = next_batch(ticket, order, nbat, &slot); b >= 0; b = next_batch(ticket, order, nbat, &slot)) {
        if (L.a[0].far_cnt) far2_batch<1>(L.a[0], b, fbuf);
        __syncthreads();  // the previous order's stage buffers are read before the next order's gathers
        if (L.a[1].far_cnt) far2_batch<2>(L.a[1], b, fbuf);
        __syncthreads();
        if (L.a[2].far_cnt) far2_batch<3>(L.a[2], b, fbuf);
        __syncthreads();
        if (L.a[3].far_cnt) far2_batch<4>(L.a[3], b, fbuf);
    }
}

// Dynamic shared memory of far_low2_kernel: the largest of its orders' stage buffers.
size_t far_low_smem() {
    return std::max(std::max(FarShape<1, float4, kFar2StageUnits>::kSmem, FarShape<2, float4, kFar2StageUnits>::kSmem),
                    std::max(FarShape<3, float4, kFar2StageUnits>::kSmem, FarShape<4, float4, kFar2StageUnits>::kSmem));
}

// The Horner scheme of `horner` with scalar coefficients.
template <int P, typename T>
__device__ __forceinline__ T horner1(const T* __restrict__ Bc, T e0, T e1, T e2, T s) {
    int q = 0;
    T G = 0;
#pragma unroll
    for (int m = (P - 1) / 2; m >= 0; --m) {
        const int Q = P - 2 * m;
        T Pp = 0;
#pragma unroll
        for (int a = Q - 1; a >= 0; --a) {
            T Qq = 0;
#pragma unroll
            for (int b = Q - 1 - a; b >= 0; --b) {
                T R = 0;
#pragma unroll
                for (int c = Q - 1 - a - b; c >= 0; --c) {
                    const T v = Bc[q++];
                    R = c == Q - 1 - a - b ? v : fma(R, e2, v);  // leading term: no FMA (see horner)
                }
                Qq = b == Q - 1 - a ? R : fma(Qq, e1, R);
            }
            Pp = a == Q - 1 ? Qq : fma(Pp, e0, Qq);
        }
        G = m == (P - 1) / 2 ? Pp : fma(G, s, Pp);
    }
    return G;
}

__device__ __forceinline__ float rsqrt_t(float x) { return rsqrtf(x); }
__device__ __forceinline__ double rsqrt_t(double x) { return rsqrt(x); }

// horner1 for two targets at once, packed across the targets (fma.rn.f32x2 with each target's own
// variable): one FMA instruction per coefficient for both targets, the same rounding per target as
// horner1.  e[t] = (e0, e1, e2, s) of target t.
template <int P>
__device__ __forceinline__ void horner1x2(const float* __restrict__ Bc, const float (&e)[2][4], float (&g)[2]) {
    int q = 0;
    float G0 = 0, G1 = 0;
#pragma unroll
    for (int m = (P - 1) / 2; m >= 0; --m) {
        const int Q = P - 2 * m;
        float P0 = 0, P1 = 0;
#pragma unroll
        for (int a = Q - 1; a >= 0; --a) {
            float Q0 = 0, Q1 = 0;
#pragma unroll
            for (int b = Q - 1 - a; b >= 0; --b) {
                float R0 = 0, R1 = 0;
#pragma unroll
                for (int c = Q - 1 - a - b; c >= 0; --c) {
                    const float v = Bc[q++];
                    if (c == Q - 1 - a - b) {
                        R0 = v; R1 = v;
                    } else {
                        fma2v(R0, R1, R0, R1, e[0][2], e[1][2], v, v);
                    }
                }
                if (b == Q - 1 - a) {
                    Q0 = R0; Q1 = R1;
                } else {
                    fma2v(Q0, Q1, Q0, Q1, e[0][1], e[1][1], R0, R1);
                }
            }
            if (a == Q - 1) {
                P0 = Q0; P1 = Q1;
            } else {
                fma2v(P0, P1, P0, P1, e[0][0], e[1][0], Q0, Q1);
            }
        }
        if (m == (P - 1) / 2) {
            G0 = P0; G1 = P1;
        } else {
            fma2v(G0, G1, G0, G1, e[0][3], e[1][3], P0, P1);
        }
    }
    g[0] = G0;
    g[1] = G1;
}

#ifndef LPM_FAR2_SCALAR_MAX_ORDER
#define LPM_FAR2_SCALAR_MAX_ORDER 12
#endif
constexpr int kFar2ScalarMaxOrder = LPM_FAR2_SCALAR_MAX_ORDER;  // FP32 scalar orders up to this: 2 targets/thread

// Far field of the scalar 1/|x - y| kernel at order P (= pm; degree < P): one block per target batch,
// T targets per thread (targets i, i + 128/T, ...; T = 2 only in FP32); each entry's contiguous
// coefficient row (stride entries, 16-byte aligned) is staged with cp.async, kK entries per stage,
// double-buffered.  Adds sum w/|x - y| to V[q].
template <int P, typename F, int T>
__global__ void __launch_bounds__(kBatch / T) far_scalar_kernel(FarArgs A, int stride) {
    constexpr int kNT = kBatch / T;
    constexpr int kU = T == 2 ? kFar2StageUnits : kFarStageUnits;
    constexpr int kE = entries_for(P);
    constexpr int kUnits = (kE * (int)sizeof(F) + 15) / 16;
    constexpr int kK = kUnits >= kU ? 1 : (kU / kUnits > 32 ? 32 : kU / kUnits);
    static_assert(T == 1 || (T == 2 && sizeof(F) == 4), "two targets per thread in FP32 only");
    extern __shared__ float4 fbuf[];  // 2 stages of kK x kUnits units, then 2 x kK centres
    double4* ctr = (double4*)(fbuf + 2 * kK * kUnits);
    __shared__ int slot;
    const int nbat = *A.nbat;
    for (int64_t b = next_batch(A.ticket, A.order, nbat, &slot); b >= 0; b = next_batch(A.ticket, A.order, nbat, &slot)) {
    const int64_t f0 = A.far_off[b], f1 = min(f0 + (int64_t)A.far_cnt[b], A.far_cap);
    if (f0 >= f1) continue;  // uniform per block
    const int64_t q0 = A.batch_first[b], qe = A.batch_first[b + 1];
    // warp w holds targets 32 T w .. 32 T (w + 1) - 1 of the batch (lane l: 32 T w + l + 32 t), so a warp past
    // the batch's last target idles as a whole
    const int64_t q = q0 + 32 * T * (threadIdx.x >> 5) + (threadIdx.x & 31);
    const bool live = q0 + 32 * T * (int64_t)(threadIdx.x >> 5) < qe;  // warp-uniform
    // T = 2 (FP32): targets and cluster centres as FP32 offsets from the batch's first target o, so that
    // d = c - x is one FP32 subtraction (the far2 kernel's scheme), and each stage's sums in FP32 folded into
    // FP64 once per stage; T = 1: FP64 positions, d rounded once from the FP64 difference
    const double4 o = A.tgt_sorted[q0];
    double4 x[T];
    float xo[T][3];
#pragma unroll
    for (int t = 0; t < T; ++t) {
        x[t] = q + 32 * t < qe ? A.tgt_sorted[q + 32 * t] : make_double4(o.x + 4.0, o.y + 4.0, o.z + 4.0, 0);
        xo[t][0] = (float)(x[t].x - o.x);
        xo[t][1] = (float)(x[t].y - o.y);
        xo[t][2] = (float)(x[t].z - o.z);
    }
    float4* ctrf = reinterpret_cast<float4*>(ctr);  // T = 2: 2 x kK FP32 centre offsets in the centres' space
    const F* base = (const F*)(sizeof(F) == 8 ? (const void*)A.B64 : (const void*)A.B32);
    auto gather = [&](int64_t s0, int n, float4* buf, int slot) {
        for (int i = threadIdx.x; i < n * kUnits; i += kNT) {
            const int e = i / kUnits, j = i - e * kUnits;
            cp_async16(buf + i, (const char*)(base + (size_t)A.far_list[s0 + e].x * stride) + 16 * j);
        }
        if ((int)threadIdx.x < n) {
            const double4 c = A.node_ctr[A.far_list[s0 + threadIdx.x].x];
            if constexpr (T == 2)
                ctrf[slot * kK + threadIdx.x] =
                    make_float4((float)(c.x - o.x), (float)(c.y - o.y), (float)(c.z - o.z), 0.0f);
            else
                ctr[slot * kK + threadIdx.x] = c;
        }
    };
    double acc[T];
#pragma unroll
    for (int t = 0; t < T; ++t) acc[t] = 0.0;
    gather(f0, (int)min((int64_t)kK, f1 - f0), fbuf, 0);
    cp_async_commit();
    int sb = 0;
    for (int64_t s0 = f0;; sb ^= 1) {
        const int n = (int)min((int64_t)kK, f1 - s0);
        const int64_t s1 = s0 + n;
        if (s1 < f1) gather(s1, (int)min((int64_t)kK, f1 - s1), fbuf + (size_t)(sb ^ 1) * kK * kUnits, sb ^ 1);
        cp_async_commit();
        cp_async_wait_prev();
        __syncthreads();  // stage sb resident
        if (live) {
            const float4* buf = fbuf + (size_t)sb * kK * kUnits;
            if constexpr (T == 2) {
                const float4* cs = ctrf + sb * kK;
                float acc32[2] = {0.0f, 0.0f};
                for (int k = 0; k < n; ++k) {
                    const float4 c = cs[k];
                    float rinv[2], e[2][4];
#pragma unroll
                    for (int t = 0; t < 2; ++t) {
                        const float dx = c.x - xo[t][0], dy = c.y - xo[t][1], dz = c.z - xo[t][2];
                        rinv[t] = rsqrt_t(dx * dx + dy * dy + dz * dz);
                        const float s2 = rinv[t] * rinv[t];
                        e[t][0] = dx * s2; e[t][1] = dy * s2; e[t][2] = dz * s2; e[t][3] = s2;
                    }
                    float g[2];
                    horner1x2<P>((const float*)(buf + (size_t)k * kUnits), e, g);
                    acc32[0] = fmaf(rinv[0], g[0], acc32[0]);
                    acc32[1] = fmaf(rinv[1], g[1], acc32[1]);
                }
                acc[0] += (double)acc32[0];
                acc[1] += (double)acc32[1];
            } else {
                const double4* cs = ctr + sb * kK;
                for (int k = 0; k < n; ++k) {
                    const F dx = (F)(cs[k].x - x[0].x), dy = (F)(cs[k].y - x[0].y), dz = (F)(cs[k].z - x[0].z);
                    const F rinv = rsqrt_t(dx * dx + dy * dy + dz * dz);
                    const F s2 = rinv * rinv;
                    const F* row = (const F*)(buf + (size_t)k * kUnits);
                    acc[0] += (double)(rinv * horner1<P, F>(row, dx * s2, dy * s2, dz * s2, s2));
                }
            }
        }
        if (s1 >= f1) break;
        __syncthreads();  // stage sb consumed before it is refilled
        s0 = s1;
    }
#pragma unroll
    for (int t = 0; t < T; ++t)
        if (q + 32 * t < qe) A.V[q + 32 * t] += acc[t];
    }
}

typedef void (*FarScalarFn)(FarArgs, int);

template <int P>
FarScalarFn far_scalar_for(bool f64, size_t* smem, int* threads) {
    constexpr int kE = entries_for(P);
    auto sm = [](int bytes, int U) {
        const int units = (kE * bytes + 15) / 16;
        const int k = units >= U ? 1 : (U / units > 32 ? 32 : U / units);
        return 2 * (size_t)k * units * 16 + 2 * (size_t)k * sizeof(double4);
    };
    *threads = kBatch;
    if (f64) {
        *smem = sm(8, kFarStageUnits);
        return far_scalar_kernel<P, double, 1>;
    }
    if constexpr (P <= kFar2ScalarMaxOrder) {
        *threads = kBatch / 2;
        *smem = sm(4, kFar2StageUnits);
        return far_scalar_kernel<P, float, 2>;
    }
    *smem = sm(4, kFarStageUnits);
    return far_scalar_kernel<P, float, 1>;
}

FarScalarFn far_scalar_select(int P, bool f64, size_t* smem, int* threads) {
    switch (P) {
        case 1: return far_scalar_for<1>(f64, smem, threads);
        case 2: return far_scalar_for<2>(f64, smem, threads);
        case 3: return far_scalar_for<3>(f64, smem, threads);
        case 4: return far_scalar_for<4>(f64, smem, threads);
        case 5: return far_scalar_for<5>(f64, smem, threads);
        case 6: return far_scalar_for<6>(f64, smem, threads);
        case 7: return far_scalar_for<7>(f64, smem, threads);
        case 8: return far_scalar_for<8>(f64, smem, threads);
        case 9: return far_scalar_for<9>(f64, smem, threads);
        case 10: return far_scalar_for<10>(f64, smem, threads);
        case 11: return far_scalar_for<11>(f64, smem, threads);
        default: return far_scalar_for<12>(f64, smem, threads);
    }
}

typedef void (*FarKernelFn)(FarArgs);

template <int P>
FarKernelFn far_kernel_for(bool f64, size_t* smem, int* threads) {
    *threads = kBatch;
    if (f64) {
        *smem = FarShape<P, double4>::kSmem;
        return far_order_kernel<P, double, double4>;
    }
    if constexpr (P <= kFar2MaxOrder) {
        *threads = kFar2Threads;
        *smem = FarShape<P, float4, kFar2StageUnits>::kSmem;
        return far_order2_kernel<P>;
    }
    *smem = FarShape<P, float4>::kSmem;
    return far_order_kernel<P, float, float4>;
}

// The two launches of the FP32 far field at kFarSplitOrder (parts 1 and 2).
FarKernelFn far_split_select(int part, size_t* smem, int* threads) {
    *threads = kFar2Threads;
    if (part == 1) {
        *smem = FarShape<kFarSplitOrder, float4, kFar2StageUnits, 1>::kSmem;
        return far_order2_kernel<kFarSplitOrder, 1>;
    }
    *smem = FarShape<kFarSplitOrder, float4, kFar2StageUnits, 2>::kSmem;
    return far_order2_kernel<kFarSplitOrder, 2>;
}

// The order-P far kernel (FP64 or FP32 arithmetic) and its dynamic shared memory.
FarKernelFn far_kernel_select(int P, bool f64, size_t* smem, int* threads) {
    switch (P) {
        case 1: return far_kernel_for<1>(f64, smem, threads);
        case 2: return far_kernel_for<2>(f64, smem, threads);
        case 3: return far_kernel_for<3>(f64, smem, threads);
        case 4: return far_kernel_for<4>(f64, smem, threads);
        case 5: return far_kernel_for<5>(f64, smem, threads);
        case 6: return far_kernel_for<6>(f64, smem, threads);
        case 7: return far_kernel_for<7>(f64, smem, threads);
        case 8: return far_kernel_for<8>(f64, smem, threads);
        case 9: return far_kernel_for<9>(f64, smem, threads);
        case 10: return far_kernel_for<10>(f64, smem, threads);
        case 11: return far_kernel_for<11>(f64, smem, threads);
        default: return far_kernel_for<12>(f64, smem, threads);
    }
}

// ---------------------------------------------------------------------------------- selector training data
// Training pairs: every `stride`-th far entry (stride <= 0: max_pairs spread over the list) -> (batch, node).
__global__ void sample_pairs_kernel(const int32_t* __restrict__ far_off, const int32_t* __restrict__ nbat,
                                    const int2* __restrict__ far_list, int64_t far_cap,
                                    const int32_t* __restrict__ totals, int64_t stride, int64_t max_pairs,
                                    int2* __restrict__ pairs, int32_t* __restrict__ n_pairs) {
    const int64_t total = min((int64_t)totals[0], far_cap);
    if (stride <= 0) stride = max((int64_t)1, (total + max_pairs - 1) / max_pairs);
    const int64_t np = min(max_pairs, (total + stride - 1) / stride);
    if (blockIdx.x == 0 && threadIdx.x == 0) *n_pairs = (int32_t)np;
    const int nb = *nbat;
    for (int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; k < np; k += (int64_t)gridDim.x * blockDim.x) {
        const int64_t f = far_off[0] + k * stride;  // far_off: the sampled order's row
        int lo = 0, hi = nb;  // last batch with far_off <= f (the one whose range holds f)
        while (hi - lo > 1) {
            const int mid = (lo + hi) >> 1;
            if (far_off[mid] <= f) lo = mid;
            else hi = mid;
        }
        pairs[k] = make_int2(lo, far_list[f].x);
    }
}

// One block per sampled (batch, cluster) pair: the cluster's exact FP64 contribution at the batch's
// targets, its expansion at orders 1..max_order (FP64), the largest per-target error of each order in
// units of |mult|, the label (smallest order within eps * sum|w|_all, else kMlpDirectClass) and the
// pair's features.
__global__ void __launch_bounds__(kBatch) label_kernel(Octree t, const int2* __restrict__ pairs,
                                                       const int32_t* __restrict__ n_pairs,
                                                       const int32_t* __restrict__ batch_first,
                                                       const double4* __restrict__ tgt_sorted,
                                                       const double4* __restrict__ src_sorted,
                                                       const double4* __restrict__ batch_ctr,
                                                       const double4* __restrict__ node_ctr,
                                                       const float* __restrict__ node_feat,
                                                       const double* __restrict__ node_wabs,
                                                       const double4* __restrict__ B64, int n_ent,
                                                       const int32_t* __restrict__ gtab, CutoffTable ct, int max_order,
                                                       double eps, float* __restrict__ feats,
                                                       int32_t* __restrict__ labels, float* __restrict__ errs) {
    extern __shared__ double4 sbuf[];
    __shared__ double red[kBatch / 32];
    const int64_t k = blockIdx.x;
    if (k >= *n_pairs) return;  // uniform per block
    const int2 pr = pairs[k];
    const int64_t q0 = batch_first[pr.x], q1 = batch_first[pr.x + 1];
    const int64_t q = q0 + threadIdx.x;
    const bool ok = q < q1;
    const double4 x = ok ? tgt_sorted[q] : make_double4(0, 0, 0, 0);
    const double4 c = node_ctr[pr.y];
    // exact contribution sum_j w_j 2 (x cross y_j) / |x - y_j|^2 (the far field's units)
    double ex[3] = {0, 0, 0};
    if (ok) {
        for (int j = t.node_start[pr.y]; j < t.node_end[pr.y]; ++j) {
            const double4 y = src_sorted[j];
            const double dx = x.x - y.x, dy = x.y - y.y, dz = x.z - y.z;
            const double s = 2.0 * y.w / (dx * dx + dy * dy + dz * dz);
            ex[0] += s * (x.y * y.z - x.z * y.y);
            ex[1] += s * (x.z * y.x - x.x * y.z);
            ex[2] += s * (x.x * y.y - x.y * y.x);
        }
    }
    const double budget = eps * node_wabs[0];
    int label = kMlpDirectClass;
    for (int P = 1; P <= max_order; ++P) {
        const int nterm = ct.table_off[P + 1] - ct.table_off[P];
        const int32_t* tab = gtab + ct.table_off[P];
        const double4* src = B64 + (size_t)pr.y * n_ent;
        __syncthreads();  // previous order's readers of sbuf / red are done
        for (int i = threadIdx.x; i < nterm; i += kBatch) sbuf[i] = src[tab[i]];
        __syncthreads();
        double v[3] = {0, 0, 0};
        far_dispatch<double, double4>(P, sbuf, x, c, v);
        double e = 0.0;
        if (ok)
            e = sqrt((v[0] - ex[0]) * (v[0] - ex[0]) + (v[1] - ex[1]) * (v[1] - ex[1]) +
                     (v[2] - ex[2]) * (v[2] - ex[2]));
        for (int o = 16; o > 0; o >>= 1) e = fmax(e, __shfl_xor_sync(0xffffffffu, e, o));
        if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = e;
        __syncthreads();
        double emax = 0.0;
        for (int i = 0; i < kBatch / 32; ++i) emax = fmax(emax, red[i]);
        if (threadIdx.x == 0 && errs) errs[k * max_order + (P - 1)] = (float)(emax / fmax(budget, 1e-300));
        if (label == kMlpDirectClass && emax <= budget) label = P - 1;
    }
    if (threadIdx.x == 0) {
        labels[k] = label;
        pair_features(batch_ctr[pr.x], c, node_feat + (size_t)pr.y * kMlpIn, log_budget(node_wabs, eps),
                      feats + k * kMlpIn);
    }
}

// ---------------------------------------------------------------------------------- near field
#ifndef LPM_NEAR_TARGETS
#define LPM_NEAR_TARGETS 2
#endif
constexpr int kNearTargets = LPM_NEAR_TARGETS;  // default targets per thread (2 or 4; run-time "near_targets")

constexpr int kNearStreamTile = 1024;  // default sources staged per tile (256, 512 or 1024; run-time "near_tile")
constexpr int kNearSplit = 2;          // default source groups per batch (1 or 2; run-time "near_split")
// The defaults (2 targets per thread, 1024 staged sources, 2 groups) were the fastest near-field shape measured
// at icos L7 and L8 (learned treecode, 512 per leaf) and within 0.4% of the fastest on 1M uniform Poisson points.
constexpr int kNearRuns = 128;        // source ranges resolved per chunk

// One tile of the stream: m tree-ordered sources (FP32 absolute coordinates, w pre-scaled by 2)
// against the thread's 2 NP targets: D += sum_j (2 w_j / |x - y_j|^2) (x - y_j), FP32 within the tile,
// FP64 across tiles.  A target's own source (d = 0) contributes 0 through the clamped denominator.
// Targets travel as packed pairs (fma.rn.f32x2): d = t - y, rr = |d|^2 + 1e-30, f = w / rr; every
// source read from shared memory serves all 2 NP targets.
template <int NP>
__device__ __forceinline__ void near_tile(const float4* tile, int m, const float (&tx)[2 * NP],
                                          const float (&ty)[2 * NP], const float (&tz)[2 * NP],
                                          double (&D)[2 * NP][3]) {
    float a[2 * NP][3];
#pragma unroll
    for (int t = 0; t < 2 * NP; ++t) a[t][0] = a[t][1] = a[t][2] = 0.f;
#pragma unroll 4
    for (int j = 0; j < m; ++j) {
        const float4 y = tile[j];
#pragma unroll
        for (int q = 0; q < NP; ++q) {
            const int t = 2 * q;
            float dx0, dx1, dy0, dy1, dz0, dz1, r0, r1;
            fma2p(dx0, dx1, y.x, y.x, -1.0f, tx[t], tx[t + 1]);
            fma2p(dy0, dy1, y.y, y.y, -1.0f, ty[t], ty[t + 1]);
            fma2p(dz0, dz1, y.z, y.z, -1.0f, tz[t], tz[t + 1]);
            fma2v(r0, r1, dx0, dx1, dx0, dx1, 1e-30f, 1e-30f);
            fma2v(r0, r1, dy0, dy1, dy0, dy1, r0, r1);
            fma2v(r0, r1, dz0, dz1, dz0, dz1, r0, r1);
            float f, g;
            fma2p(f, g, rcp32(r0), rcp32(r1), y.w, -0.0f, -0.0f);  // w / rr for both targets in one instruction
            fma2v(a[t][0], a[t + 1][0], f, g, dx0, dx1, a[t][0], a[t + 1][0]);
            fma2v(a[t][1], a[t + 1][1], f, g, dy0, dy1, a[t][1], a[t + 1][1]);
            fma2v(a[t][2], a[t + 1][2], f, g, dz0, dz1, a[t][2], a[t + 1][2]);
        }
    }
#pragma unroll
    for (int t = 0; t < 2 * NP; ++t) {
        D[t][0] += a[t][0];
        D[t][1] += a[t][1];
        D[t][2] += a[t][2];
    }
}

// Biot-Savart: the result of target q (sorted order), u = mult (V - x cross D), the far field V complete.
__device__ __forceinline__ void finish_target(int64_t q, int64_t qe, int64_t n_tgt, const double4& x,
                                              const double* D, const int32_t* __restrict__ tperm,
                                              const double* __restrict__ V, double mult, double* __restrict__ U) {
    if (q >= qe) return;
    const double v0 = V[q], v1 = V[n_tgt + q], v2 = V[2 * n_tgt + q];
    const int64_t o = tperm[q];
    U[o] = mult * (v0 - (x.y * D[2] - x.z * D[1]));
    U[n_tgt + o] = mult * (v1 - (x.z * D[0] - x.x * D[2]));
    U[2 * n_tgt + o] = mult * (v2 - (x.x * D[1] - x.y * D[0]));
}

// A batch's near work is the concatenation of its source ranges (runs of consecutive leaves, then
// clusters whose order was set to "direct"); it is streamed through shared memory in tiles of
// kNearStreamTile sources regardless of how short the individual ranges are.
// One tile of the scalar 1/r stream: D += sum_j w_j / |x - y_j| (FP32 within the tile, FP64 across
// tiles); a source at the target's own position (r = 0) contributes nothing.  Pairs of targets packed as
// in near_tile.
template <int NP>
__device__ __forceinline__ void near_tile_scalar(const float4* tile, int m, const float (&tx)[2 * NP],
                                                 const float (&ty)[2 * NP], const float (&tz)[2 * NP],
                                                 double (&D)[2 * NP][3]) {
    float a[2 * NP];
#pragma unroll
    for (int t = 0; t < 2 * NP; ++t) a[t] = 0.f;
#pragma unroll 4
    for (int j = 0; j < m; ++j) {
        const float4 y = tile[j];
#pragma unroll
        for (int q = 0; q < NP; ++q) {
            const int t = 2 * q;
            float dx0, dx1, dy0, dy1, dz0, dz1, r0, r1;
            fma2p(dx0, dx1, y.x, y.x, -1.0f, tx[t], tx[t + 1]);
            fma2p(dy0, dy1, y.y, y.y, -1.0f, ty[t], ty[t + 1]);
            fma2p(dz0, dz1, y.z, y.z, -1.0f, tz[t], tz[t + 1]);
            fma2v(r0, r1, dx0, dx1, dx0, dx1, -0.0f, -0.0f);
            fma2v(r0, r1, dy0, dy1, dy0, dy1, r0, r1);
            fma2v(r0, r1, dz0, dz1, dz0, dz1, r0, r1);
            const float i0 = r0 > 0.f ? rsqrt32(r0) : 0.f, i1 = r1 > 0.f ? rsqrt32(r1) : 0.f;
            fma2p(a[t], a[t + 1], i0, i1, y.w, a[t], a[t + 1]);
        }
    }
#pragma unroll
    for (int t = 0; t < 2 * NP; ++t) D[t][0] += a[t];
}

__device__ __forceinline__ void finish_target_scalar(int64_t q, int64_t qe, const double* D, double* __restrict__ W) {
    if (q >= qe) return;
    W[q] = D[0];  // far_near_combine_kernel forms u = mult (V + W)
}

// Scalar kernel: the result in the caller's target order, u = mult (V + W), V the far field's sum and W the near
// field's, both in sorted order.  The near and far kernels write disjoint buffers, so they run concurrently.
__global__ void far_near_combine_kernel(const double* __restrict__ V, const double* __restrict__ W,
                                        const int32_t* __restrict__ tperm, int64_t n, double mult,
                                        double* __restrict__ U) {
    for (int64_t q = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; q < n; q += (int64_t)gridDim.x * blockDim.x)
        U[tperm[q]] = mult * (V[q] + W[q]);
}

struct NearArgs {
    Octree t;
    const double4* tgt_sorted;
    int64_t n_tgt;
    const int32_t* batch_first;
    const int32_t* nbat;
    const int32_t* near_off;
    const int32_t* near_cnt;
    const int2* near_list;
    int64_t near_cap;
    const float4* src32;
    double* W;  // scalar kernel: near-field output per sorted target
    // Biot-Savart: the result u = mult (V - x cross D) in the caller's target order
    const int32_t* tperm;
    const double* V;
    double mult;
    double* U;
    const int32_t* order;  // batches in decreasing order of near work
    int32_t* ticket;       // zeroed before the launch
};

// One batch b of the near kernel (the whole block).
// Tile shape: KT targets per thread and KTILE sources staged in shared memory per tile; KS groups of
// kBatch / KT threads each hold the whole batch and sum their own contiguous share of every tile (KS = 2
// gives each source read from shared memory to KT targets while keeping two warps on a batch), and the
// groups' sums are added in shared memory at the end of the batch.  Instances for KT in {2, 4}, KTILE in
// {256, 512, 1024} and KS in {1, 2} are chosen at run time.
template <bool kScalar, int KT, int KTILE, int KS>
__device__ __forceinline__ void near_batch(const NearArgs& A, int64_t b) {
    constexpr int kT = KT, kTT = kBatch / KT, kThreads = kTT * KS, kNW = kThreads / 32, kRPT = kNearRuns / kThreads;
    static_assert(kT % 2 == 0 && kTT % 32 == 0 && kNearRuns % kThreads == 0, "near kernel shape");
    static_assert((KS - 1) * 3 * kBatch * sizeof(double) <= sizeof(float4) * KTILE, "group sums fit one tile");
    __shared__ __align__(16) float4 tile[2][KTILE];  // double-buffered: tile p + 1 arrives while p is summed
    __shared__ int r_start[kNearRuns], r_pre[kNearRuns + 1];
    __shared__ int warp_tot[kNW];
    const Octree& t = A.t;
    const double4* __restrict__ tgt_sorted = A.tgt_sorted;
    const int32_t* __restrict__ batch_first = A.batch_first;
    const int32_t* __restrict__ near_off = A.near_off;
    const int32_t* __restrict__ near_cnt = A.near_cnt;
    const int2* __restrict__ near_list = A.near_list;
    const float4* __restrict__ src32 = A.src32;
    const int64_t near_cap = A.near_cap;
    const int64_t qe = batch_first[b + 1];
    // within each group, warp w holds targets 32 kT w .. 32 kT (w + 1) - 1 of the batch (lane l: 32 kT w + l +
    // 32 u), so a warp past the batch's last target skips the arithmetic as a whole
    const int tid = (int)threadIdx.x % kTT, part = (int)threadIdx.x / kTT;
    const int64_t qw = batch_first[b] + 32 * kT * (tid >> 5) + (tid & 31);
    const bool live = batch_first[b] + 32 * kT * (int64_t)(tid >> 5) < qe;  // warp-uniform
    float tx[kT], ty[kT], tz[kT];
    double D[kT][3];
#pragma unroll
    for (int u = 0; u < kT; ++u) {
        const int64_t q = qw + 32 * u;
        const double4 x = q < qe ? tgt_sorted[q] : make_double4(2, 2, 2, 0);
        tx[u] = (float)x.x;
        ty[u] = (float)x.y;
        tz[u] = (float)x.z;
        D[u][0] = D[u][1] = D[u][2] = 0.0;
    }
    const int64_t n0 = near_off[b], n1 = min(n0 + (int64_t)near_cnt[b], near_cap);
    const int64_t n_all = n1 - n0;
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    for (int64_t c0 = 0; c0 < n_all; c0 += kNearRuns) {
        // resolve up to kNearRuns entries into source ranges and their prefix offsets
        int len[kRPT], st[kRPT];
        int v = 0;
#pragma unroll
        for (int h = 0; h < kRPT; ++h) {
            const int64_t k = c0 + threadIdx.x * kRPT + h;
            len[h] = 0;
            st[h] = 0;
            if (k < n_all) {
                const int2 r = near_list[n0 + k];
                st[h] = t.node_start[t.leaf_node[r.x]];
                len[h] = t.node_end[t.leaf_node[r.y]] - st[h];
            }
            v += len[h];
        }
        // exclusive scan of the kNearRuns lengths (kNW warps)
        int incl = v;
        for (int o = 1; o < 32; o <<= 1) {
            const int u = __shfl_up_sync(0xffffffffu, incl, o);
            if (lane >= o) incl += u;
        }
        __syncthreads();  // previous chunk's readers of r_pre / r_start / tile are done
        if (lane == 31) warp_tot[w] = incl;
        __syncthreads();
        int base = incl - v, total = 0;
#pragma unroll
        for (int k = 0; k < kNW; ++k) {
            if (k < w) base += warp_tot[k];
            total += warp_tot[k];
        }
#pragma unroll
        for (int h = 0; h < kRPT; ++h) {
            r_pre[threadIdx.x * kRPT + h] = base;
            r_start[threadIdx.x * kRPT + h] = st[h];
            base += len[h];
        }
        if (threadIdx.x == 0) r_pre[kNearRuns] = total;
        __syncthreads();
        // the sources of positions p0 .. p0 + KTILE - 1 of the chunk's stream go to tile[buf] by asynchronous
        // copies (the run holding position p found by binary search of the prefix offsets)
        auto stage = [&](int p0, int buf) {
            const int m = min(KTILE, total - p0);
            int lo = 0;
            for (int j = threadIdx.x; j < m; j += kThreads) {
                const int p = p0 + j;
                int hi = kNearRuns;  // last run r with r_pre[r] <= p (positions grow: search from the last one)
                while (hi - lo > 1) {
                    const int mid = (lo + hi) >> 1;
                    if (r_pre[mid] <= p) lo = mid;
                    else hi = mid;
                }
                cp_async16(&tile[buf][j], src32 + r_start[lo] + (p - r_pre[lo]));
            }
        };
        int buf = 0;
        if (total > 0) stage(0, 0);
        cp_async_commit();
        for (int p0 = 0; p0 < total; p0 += KTILE, buf ^= 1) {
            const int m = min(KTILE, total - p0);
            if (p0 + KTILE < total) stage(p0 + KTILE, buf ^ 1);
            cp_async_commit();
            cp_async_wait_prev();  // this thread's copies into tile[buf] have landed
            __syncthreads();       // ... and every other thread's
            if (live) {
                const int h = (m + KS - 1) / KS, lo = min(m, part * h), cnt = min(m - lo, h);  // this group's share
                if constexpr (kScalar)
                    near_tile_scalar<kT / 2>(tile[buf] + lo, cnt, tx, ty, tz, D);
                else
                    near_tile<kT / 2>(tile[buf] + lo, cnt, tx, ty, tz, D);
            }
            __syncthreads();  // tile[buf] is read before the next stage refills it
        }
    }
    if constexpr (KS > 1) {  // add the other groups' sums to group 0's through the (consumed) tile buffer
        double* red = reinterpret_cast<double*>(&tile[0][0]);
        __syncthreads();
        if (part > 0)
#pragma unroll
            for (int u = 0; u < kT; ++u)
#pragma unroll
                for (int c = 0; c < 3; ++c) red[(((part - 1) * kT + u) * 3 + c) * kTT + tid] = D[u][c];
        __syncthreads();
        if (part > 0) return;  // block-uniform barriers follow only in next_batch
#pragma unroll
        for (int g = 1; g < KS; ++g)
#pragma unroll
            for (int u = 0; u < kT; ++u)
#pragma unroll
                for (int c = 0; c < 3; ++c) D[u][c] += red[(((g - 1) * kT + u) * 3 + c) * kTT + tid];
    }
#pragma unroll
    for (int u = 0; u < kT; ++u) {
        const int64_t q = qw + 32 * u;
        if constexpr (kScalar)
            finish_target_scalar(q, qe, D[u], A.W);
        else if (q < qe)
            finish_target(q, qe, A.n_tgt, tgt_sorted[q], D[u], A.tperm, A.V, A.mult, A.U);  // FP64 x re-read
    }
}

// Persistent: every block takes batches from the ticket in `order` until none is left; one batch at a time
// through near_batch.
template <bool kScalar, int KT, int KTILE, int KS>
__global__ void __launch_bounds__(kBatch / KT * KS) near_kernel(NearArgs A) {
    __shared__ int slot;
    const int nbat = *A.nbat;
    for (int64_t b = next_batch(A.ticket, A.order, nbat, &slot); b >= 0; b = next_batch(A.ticket, A.order, nbat, &slot))
        near_batch<kScalar, KT, KTILE, KS>(A, b);
}

typedef void (*NearFn)(NearArgs);

// The near kernel of a tile shape (targets per thread 2 or 4; staged sources 256, 512 or 1024; 1 or 2
// source groups) and its block size; nullptr for another shape.
NearFn near_select(bool scalar, int targets, int tile, int split, int* threads) {
    *threads = kBatch / targets * split;
#define LPM_NEAR_CASE(T, TILE, S)                                     \
    if (targets == T && tile == TILE && split == S)                    \
        return scalar ? near_kernel<true, T, TILE, S> : near_kernel<false, T, TILE, S>;
    LPM_NEAR_CASE(2, 256, 1)
    LPM_NEAR_CASE(2, 512, 1)
    LPM_NEAR_CASE(2, 1024, 1)
    LPM_NEAR_CASE(4, 256, 1)
    LPM_NEAR_CASE(4, 512, 1)
    LPM_NEAR_CASE(4, 1024, 1)
    LPM_NEAR_CASE(2, 256, 2)
    LPM_NEAR_CASE(2, 512, 2)
    LPM_NEAR_CASE(2, 1024, 2)
    LPM_NEAR_CASE(4, 256, 2)
    LPM_NEAR_CASE(4, 512, 2)
    LPM_NEAR_CASE(4, 1024, 2)
#undef LPM_NEAR_CASE
    return nullptr;
}

// ---------------------------------------------------------------------------------- fused solvers
// The far and near fields of many solvers' evaluations (an ensemble's instances at one RK4 stage) in one
// persistent launch per far order and per near tile shape.  The work items are the (solver, batch) pairs of
// every solver, bucketed by decreasing work over all of them, so that a launch ends on the smallest batches of
// any solver; a block copies its item's solver arguments to shared memory and runs the per-batch body of the
// solver's own launch, so every batch is summed exactly as there (bitwise the same results).
struct FusedSched {
    const int2* items;     // (solver, batch) by decreasing work over all solvers
    const int32_t* total;  // number of items
    int32_t* ticket;       // zeroed before the launch
};
struct FusedInst {
    const uint32_t* far_work;
    const uint32_t* near_work;
    const int32_t* nbat;  // the solver's batch count; null: the solver takes no part
};
constexpr int kFusedFarSlots = kPMax + 2;  // slot P: order P; slot kPMax + 1: part 2 of kFarSplitOrder
constexpr int kFusedNearGroups = 12;       // near tile shapes
// fused schedule scratch (int32): far buckets and cursors, near buckets and cursors, the two item counts, one
// ticket per far slot and one per near group
constexpr int kFzFarHist = 0, kFzFarCur = 64, kFzNearHist = 128, kFzNearCur = 192, kFzTotals = 256,
              kFzFarTicket = 258, kFzNearTicket = kFzFarTicket + kFusedFarSlots,
              kFzInts = kFzNearTicket + kFusedNearGroups;

// grid (x, solvers); the buckets are zeroed by the caller.
__global__ void fused_hist_kernel(const FusedInst* __restrict__ inst, int32_t* __restrict__ aux) {
    const FusedInst I = inst[blockIdx.y];
    const int n = I.nbat ? *I.nbat : 0;
    for (int b = blockIdx.x * blockDim.x + threadIdx.x; b < n; b += gridDim.x * blockDim.x) {
        atomicAdd(&aux[kFzFarHist + sched_bucket(I.far_work[b])], 1);
        atomicAdd(&aux[kFzNearHist + sched_bucket(I.near_work[b])], 1);
    }
}

__global__ void fused_scatter_kernel(const FusedInst* __restrict__ inst, int32_t* __restrict__ aux,
                                     int2* __restrict__ far_items, int2* __restrict__ near_items) {
    __shared__ int fbase[kSchedBuckets], nbase[kSchedBuckets];
    if (threadIdx.x == 0) {
        int fa = 0, na = 0;
        for (int k = 0; k < kSchedBuckets; ++k) {
            fbase[k] = fa;
            fa += aux[kFzFarHist + k];
            nbase[k] = na;
            na += aux[kFzNearHist + k];
        }
        if (blockIdx.x == 0 && blockIdx.y == 0) {
            aux[kFzTotals] = fa;
            aux[kFzTotals + 1] = na;
        }
    }
    __syncthreads();
    const FusedInst I = inst[blockIdx.y];
    const int n = I.nbat ? *I.nbat : 0;
    for (int b = blockIdx.x * blockDim.x + threadIdx.x; b < n; b += gridDim.x * blockDim.x) {
        const int kf = sched_bucket(I.far_work[b]), kn = sched_bucket(I.near_work[b]);
        far_items[fbase[kf] + atomicAdd(&aux[kFzFarCur + kf], 1)] = make_int2((int)blockIdx.y, b);
        near_items[nbase[kn] + atomicAdd(&aux[kFzNearCur + kn], 1)] = make_int2((int)blockIdx.y, b);
    }
}

// Whether a fused launch computes item (solver, b): the solver takes part in it and, for a far order, has
// clusters of that order in batch b (a near item always writes its targets' result).
__device__ __forceinline__ bool fused_has_work(const FarArgs& a, int b) {
    return a.far_cnt != nullptr && a.far_cnt[b] > 0;
}
__device__ __forceinline__ bool fused_has_work(const NearArgs& a, int) { return a.near_cnt != nullptr; }

// The block's next item of a fused launch, with its solver's arguments copied to araw; false when none is left.
template <typename Args>
__device__ __forceinline__ bool next_fused_item(const FusedSched& S, int n, const Args* __restrict__ tab,
                                                uint32_t* araw, int2* item) {
    __syncthreads();  // every thread is done with the previous item's shared memory
    if (threadIdx.x == 0) {
        int2 v = make_int2(-1, -1);
        for (int k = atomicAdd(S.ticket, 1); k < n; k = atomicAdd(S.ticket, 1)) {
            const int2 c = S.items[k];
            if (fused_has_work(tab[c.x], c.y)) {
                v = c;
                break;
            }
        }
        *item = v;
    }
    __syncthreads();
    const int2 v = *item;
    if (v.x < 0) return false;
    const uint32_t* src = reinterpret_cast<const uint32_t*>(tab + v.x);
    for (int w = threadIdx.x; w < (int)(sizeof(Args) / 4); w += blockDim.x) araw[w] = src[w];
    __syncthreads();
    return true;
}

// far_order2_kernel over the items of many solvers: tab[s] holds solver s's arguments for this order (part).
template <int P, int PART = 0>
__global__ void __launch_bounds__(kFar2Threads, kFar2MinBlocks) far_fused2_kernel(const FarArgs* __restrict__ tab,
                                                                                  FusedSched S) {
    static_assert(sizeof(FarArgs) % 4 == 0, "argument copy by words");
    extern __shared__ float4 fbuf[];
    __shared__ __align__(16) uint32_t araw[sizeof(FarArgs) / 4];
    __shared__ int2 item;
    const FarArgs& A = *reinterpret_cast<const FarArgs*>(araw);
    const int n = *S.total;
    while (next_fused_item(S, n, tab, araw, &item)) far2_batch<P, PART>(A, item.y, fbuf);
}

// near_kernel (Biot-Savart) over the items of many solvers sharing one tile shape.
template <int KT, int KTILE, int KS>
__global__ void __launch_bounds__(kBatch / KT * KS) near_fused_kernel(const NearArgs* __restrict__ tab, FusedSched S) {
    static_assert(sizeof(NearArgs) % 4 == 0, "argument copy by words");
    __shared__ __align__(16) uint32_t araw[sizeof(NearArgs) / 4];
    __shared__ int2 item;
    const NearArgs& A = *reinterpret_cast<const NearArgs*>(araw);
    const int n = *S.total;
    while (next_fused_item(S, n, tab, araw, &item)) near_batch<false, KT, KTILE, KS>(A, item.y);
}

typedef void (*FarFusedFn)(const FarArgs*, FusedSched);
typedef void (*NearFusedFn)(const NearArgs*, FusedSched);

// The fused far kernel of FP32 order P (1..kFar2MaxOrder; part 1 or 2 at kFarSplitOrder, else 0).
template <int P>
FarFusedFn far_fused_for(int part, size_t* smem) {
    if constexpr (P == kFarSplitOrder) {
        if (part == 2) {
            *smem = FarShape<P, float4, kFar2StageUnits, 2>::kSmem;
            return far_fused2_kernel<P, 2>;
        }
        *smem = FarShape<P, float4, kFar2StageUnits, 1>::kSmem;
        return far_fused2_kernel<P, 1>;
    } else {
        *smem = FarShape<P, float4, kFar2StageUnits>::kSmem;
        return far_fused2_kernel<P>;
    }
}
FarFusedFn far_fused_select(int P, int part, size_t* smem, int* threads) {
    static_assert(kFar2MaxOrder == 11 && kFarSplitOrder == 11, "fused far orders 1..11");
    *threads = kFar2Threads;
    switch (P) {
        case 1: return far_fused_for<1>(part, smem);
        case 2: return far_fused_for<2>(part, smem);
        case 3: return far_fused_for<3>(part, smem);
        case 4: return far_fused_for<4>(part, smem);
        case 5: return far_fused_for<5>(part, smem);
        case 6: return far_fused_for<6>(part, smem);
        case 7: return far_fused_for<7>(part, smem);
        case 8: return far_fused_for<8>(part, smem);
        case 9: return far_fused_for<9>(part, smem);
        case 10: return far_fused_for<10>(part, smem);
        case 11: return far_fused_for<11>(part, smem);
        default: return nullptr;
    }
}

NearFusedFn near_fused_select(int targets, int tile, int split, int* threads) {
    *threads = kBatch / targets * split;
#define LPM_NEAR_FUSED_CASE(T, TILE, S) \
    if (targets == T && tile == TILE && split == S) return near_fused_kernel<T, TILE, S>;
    LPM_NEAR_FUSED_CASE(2, 256, 1)
    LPM_NEAR_FUSED_CASE(2, 512, 1)
    LPM_NEAR_FUSED_CASE(2, 1024, 1)
    LPM_NEAR_FUSED_CASE(4, 256, 1)
    LPM_NEAR_FUSED_CASE(4, 512, 1)
    LPM_NEAR_FUSED_CASE(4, 1024, 1)
    LPM_NEAR_FUSED_CASE(2, 256, 2)
    LPM_NEAR_FUSED_CASE(2, 512, 2)
    LPM_NEAR_FUSED_CASE(2, 1024, 2)
    LPM_NEAR_FUSED_CASE(4, 256, 2)
    LPM_NEAR_FUSED_CASE(4, 512, 2)
    LPM_NEAR_FUSED_CASE(4, 1024, 2)
#undef LPM_NEAR_FUSED_CASE
    return nullptr;
}

// host-side tables --------------------------------------------------------------------------------
void canonical_entries(int pm, std::vector<int4>& ent) {
    ent.clear();
    for (int m = (pm - 1) / 2; m >= 0; --m) {
        const int Q = pm - 2 * m;
        for (int a = Q - 1; a >= 0; --a)
            for (int b = Q - 1 - a; b >= 0; --b)
                for (int c = Q - 1 - a - b; c >= 0; --c) ent.push_back(make_int4(m, a, b, c));
    }
}

}  // namespace

// Cost model: an order-P expansion costs ~8 E(P) + 40 flops per target (twice that in FP64), a
// direct pair 17; a cluster with fewer sources than this is cheaper to sum directly.

static int32_t direct_cutoff(int P, int f64_from, bool scalar) {
    // scalar 1/r: 2 flops per coefficient + ~12 of setup against 11 per direct pair
    if (scalar) return (int32_t)((P >= f64_from ? 2.0 : 1.0) * (2.0 * entries_for(P) + 12.0) / 11.0);
    return (int32_t)((P >= f64_from ? 2.0 : 1.0) * (8.0 * entries_for(P) + 40.0) / 17.0);
}

struct TreeSolver {
    lpm_ctx* ctx = nullptr;
    lpm_kernel_desc kernel{};
    lpm_solver_desc solver{};
    int64_t n_src = 0, n_tgt = 0;
    int64_t n_batches = 0;  // capacity: launch size of the per-batch kernels
    int batch_level = 1;    // octree level whose cells batches may not straddle
    int batch_level_max = 1;  // the level the batch capacity was sized for (finest allowed)
    int32_t* bflag = nullptr;
    int32_t* batch_first = nullptr;
    int pm = 8;
    int order = 8;         // the fixed order in the internal convention (degree < order)
    bool scalar = false;   // the 1/(4 pi r) kernel (else Biot-Savart on the sphere)
    int a_stride = 0;      // scalar kernel: coefficient row length (padded to 4 entries)
    double* A64 = nullptr;  // scalar kernel: coefficient rows (FP64, FP32)
    float* A32 = nullptr;
    int f64_from = kF64From;  // far expansions of order >= f64_from evaluate in FP64
    int heavy_cap = 0;        // nodes the moment / coefficient / feature arrays hold (grown on demand)
    // root box of the source octree: Box3d(R) padded by 1e-5 (src/LpmBox3d.h:21-33).  Biot-Savart: R is
    // root_maxr when positive, else maxR (src/LpmCoords.cpp:136-143) of targets[root_first:n_tgt] computed on
    // the device (TreeSum's mesh constructor takes maxR of the mesh vertices, src/LpmTreeSum.cpp:227; the RK4
    // integrator points root_first at its vertex particles), or of the sources when that range is empty.
    // Poisson: R is the largest |coordinate| of the sources (the smallest such cube holding them).
    double root_maxr = 0.0;
    int64_t root_first = 0;
    unsigned long long* root_r = nullptr;
    Octree st;
    // target ordering
    uint64_t* tkeys = nullptr;
    int32_t* tperm = nullptr;
    uint64_t* ttmpk = nullptr;
    int32_t* ttmpv = nullptr;
    int32_t* tcount = nullptr;
    double4* tgt_sorted = nullptr;
    double4* batch_ctr = nullptr;
    // sources and nodes
    double4* src_sorted = nullptr;
    float4* src32 = nullptr;
    double4* node_ctr = nullptr;
    double* node_wabs = nullptr;
    double* node_mom = nullptr;
    double4* B64 = nullptr;
    float4* B32 = nullptr;
    int n_ent = 0;
    int4* ent = nullptr;
    int4* mono = nullptr;
    int4* p2m_units = nullptr;  // leaf moment units (a, b, c0)
    int32_t* m2m_pending = nullptr;  // per node: internal children whose moments are not yet shifted
    int n_units = 0;
    int n_mono = 0;
    int32_t* gtab = nullptr;
    CutoffTable ct{};
    // interaction lists
    int32_t *far_cnt = nullptr, *near_cnt = nullptr, *far_off = nullptr, *near_off = nullptr, *flags = nullptr;
    unsigned long long* pair_counts = nullptr;
    int2 *far_list = nullptr, *near_list = nullptr;
    int64_t far_cap = 0, near_cap = 0;
    double* V = nullptr;
    double* W = nullptr;              // near-field output (sorted targets), combined with V into the result
    // the near field runs on `side` beside the far-field launches on the context's stream (fork / join events)
    cudaStream_t side = nullptr;
    cudaEvent_t ev_fork = nullptr, ev_join = nullptr;
    cudaEvent_t ev_tfork = nullptr, ev_tjoin = nullptr;  // target batches on `side` beside the tree build
    cudaEvent_t ev_cfork = nullptr, ev_cjoin = nullptr;  // far coefficients on `side` beside the traversal
    // learned order selection
    bool learned = false;     // order_policy == LPM_ORDER_LEARNED
    bool mlp_loaded = false;  // weights present; without them the fixed order is the fallback
    double eps = 2e-8;        // per-pair error budget relative to |mult| * sum|w|
    int order_bias = 0;       // orders added to the selector's choice
    float* node_feat = nullptr;
    __nv_bfloat16* mlp_w = nullptr;
    float* mlp_norm = nullptr;
    uint8_t* decisions = nullptr;  // selector decisions of the count pass, reused by the fill pass
    // batch schedules of the persistent near and far kernels
    uint32_t* near_work = nullptr;    // per batch: near-field pairs (count pass)
    uint32_t* far_work = nullptr;     // per batch: far coefficient evaluations (count pass)
    int32_t* sched_order = nullptr;   // batches by decreasing near work
    int32_t* far_order = nullptr;     // batches by decreasing far work
    int32_t* sched_aux = nullptr;     // kAux* layout below
    int near_blocks = 1;              // persistent grids: resident blocks on the whole device
    int near_targets = kNearTargets;  // near kernel tile shape (run-time "near_targets", "near_tile")
    int near_tile = kNearStreamTile;
    int near_split = kNearSplit;      // source groups per batch (run-time "near_split")
    int far_blocks[kPMax + 1][2] = {};  // per order, FP32 / FP64 far kernel
    int far_split_blocks[2] = {};       // the two FP32 launches of order kFarSplitOrder
    int far_low_blocks = 1;             // far_low2_kernel (FP32 orders 1..kFarLowMax in one launch)
    uint64_t generation = 0;          // reallocations of the lists and per-node arrays (tree_generation)
    std::vector<void*> allocs;
};

// Dynamic shared memory of every far kernel above 48 KB needs the opt-in attribute.
static cudaError_t far_smem_attributes() {
    for (int P = 1; P <= kPMax; ++P)
        for (int f64 = 0; f64 < 2; ++f64) {
            size_t smem = 0;
            int threads = 0;
            FarKernelFn fn = far_kernel_select(P, f64 != 0, &smem, &threads);
            if (smem > 48 * 1024) {
                const cudaError_t e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
                if (e != cudaSuccess) return e;
            }
        }
    return cudaSuccess;
}

namespace {

template <typename Tp>
cudaError_t talloc(TreeSolver* t, Tp** p, size_t count) {
    cudaError_t e = dev_alloc((void**)p, std::max<size_t>(count, 1) * sizeof(Tp));
    if (e == cudaSuccess) t->allocs.push_back(*p);
    return e;
}

int alloc_lists(TreeSolver* t, int64_t far_cap, int64_t near_cap) {
    for (void** p : {(void**)&t->far_list, (void**)&t->near_list}) {
        if (*p) {
            cudaFree(*p);
            t->allocs.erase(std::find(t->allocs.begin(), t->allocs.end(), *p));
            *p = nullptr;
        }
    }
    ++t->generation;
    cudaError_t e = talloc(t, &t->far_list, (size_t)far_cap);
    if (e == cudaSuccess) e = talloc(t, &t->near_list, (size_t)near_cap);
    if (e != cudaSuccess) return cuda_status(e, "cudaMalloc (interaction lists)");
    t->far_cap = far_cap;
    t->near_cap = near_cap;
    return LPM_OK;
}

// Regrow the per-node moment / coefficient / feature arrays to hold `need` nodes (with headroom).
int heavy_alloc(TreeSolver* t, int64_t need) {
    const int64_t cap = std::min<int64_t>(t->st.node_cap, need + need / 2 + 256);
    auto regrow = [&](auto** p, size_t per_node) -> cudaError_t {
        if (*p) {
            cudaFree(*p);
            t->allocs.erase(std::find(t->allocs.begin(), t->allocs.end(), (void*)*p));
            *p = nullptr;
        }
        return talloc(t, p, (size_t)cap * per_node);
    };
    ++t->generation;
    cudaError_t e = regrow(&t->node_mom, (size_t)mono_count(t->pm));
    if (e == cudaSuccess && t->scalar) e = regrow(&t->A64, (size_t)t->a_stride);
    if (e == cudaSuccess && t->scalar) e = regrow(&t->A32, (size_t)t->a_stride);
    if (e == cudaSuccess && !t->scalar) e = regrow(&t->B64, (size_t)t->n_ent);
    if (e == cudaSuccess && !t->scalar) e = regrow(&t->B32, (size_t)t->n_ent);
    if (e == cudaSuccess && t->learned) e = regrow(&t->node_feat, (size_t)kMlpIn);
    if (e != cudaSuccess) return cuda_status(e, "cudaMalloc (node moments)");
    t->heavy_cap = (int)cap;
    return LPM_OK;
}

std::mutex constants_mu;
uint64_t constants_ready = 0;  // bit d: device d holds the tables

int upload_constants() {
    int dev = 0;
    LPM_CUDA_TRY(cudaGetDevice(&dev));
    std::lock_guard<std::mutex> lock(constants_mu);
    if (dev < 64 && ((constants_ready >> dev) & 1)) return LPM_OK;
    double binom[kPMax + 2][kPMax + 2] = {};
    for (int n = 0; n < kPMax + 2; ++n) {
        binom[n][0] = 1.0;
        for (int k = 1; k <= n; ++k) binom[n][k] = binom[n - 1][k - 1] + (k <= n - 1 ? binom[n - 1][k] : 0.0);
    }
    double fact[2 * kPMax + 2];
    fact[0] = 1.0;
    for (int i = 1; i < 2 * kPMax + 2; ++i) fact[i] = fact[i - 1] * i;
    LPM_CUDA_TRY(cudaMemcpyToSymbol(c_binom, binom, sizeof(binom)));
    LPM_CUDA_TRY(cudaMemcpyToSymbol(c_fact, fact, sizeof(fact)));
    if (dev < 64) constants_ready |= 1ull << dev;
    return LPM_OK;
}

}  // namespace

// Select the near kernel's tile shape and size its persistent grid (resident blocks on the device).
static int near_shape(TreeSolver* t, int targets, int tile, int split) {
    int threads = 0;
    NearFn fn = near_select(t->scalar, targets, tile, split, &threads);
    if (!fn) {
        set_error("tree solver: near_targets must be 2 or 4, near_tile 256, 512 or 1024 and near_split 1 or 2");
        return LPM_ERR_ARG;
    }
    int per_sm = 0;
    LPM_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fn, threads, 0));
    t->near_targets = targets;
    t->near_tile = tile;
    t->near_split = split;
    t->near_blocks = (int)std::max<int64_t>(1, std::min<int64_t>(t->n_batches,
                                                                  (int64_t)std::max(per_sm, 1) * t->ctx->num_sms));
    return LPM_OK;
}

int tree_solver_create(lpm_ctx* ctx, const lpm_kernel_desc& kernel, const lpm_solver_desc& solver, int64_t n_src,
                       int64_t n_tgt, TreeSolver** out) {
    *out = nullptr;
    const bool scalar = kernel.kind == LPM_KERNEL_POISSON_3D;
    if (!scalar && (kernel.kind != LPM_KERNEL_BIOT_SAVART_SPHERE || kernel.radius != 1.0 || kernel.delta != 0.0)) {
        set_error("tree solver: supports the singular Biot-Savart kernel on the unit sphere and the 3D Poisson kernel");
        return LPM_ERR_KERNEL;
    }
    // Biot-Savart: order p = multi-indices |k| < p (the reference's SumNode); Poisson: |k| <= p (the
    // reference's TaylorSeries3d convention), i.e. internal order p + 1
    const int order = scalar ? solver.order + 1 : solver.order;
    const int sakajo = solver.sakajo_depth;
    if (order < 1 || order > kPMax || (sakajo == 0 && solver.max_per_leaf < 1) || !(solver.theta > 0.0) ||
        solver.theta >= 1.0 || n_src >= INT32_MAX || n_tgt >= INT32_MAX || sakajo < 0 || 3 * sakajo > kMaxLevels) {
        set_error("tree solver: need 1 <= order <= %d (Poisson: 0 <= order <= %d), max_per_leaf >= 1 (octree) or "
                  "1 <= sakajo_depth <= 21, 0 < theta < 1", kPMax, kPMax - 1);
        return LPM_ERR_ARG;
    }
    if (sakajo > 0 && scalar) {
        set_error("tree solver: the Sakajo tree is built for the sphere (Biot-Savart kernel)");
        return LPM_ERR_ARG;
    }
    if (scalar && solver.order_policy == LPM_ORDER_LEARNED) {
        set_error("tree solver: the learned order selector is trained for the Biot-Savart kernel only");
        return LPM_ERR_ARG;
    }
    int rc = upload_constants();
    if (rc) return rc;
    TreeSolver* t = new (std::nothrow) TreeSolver();
    if (!t) return LPM_ERR_OOM;
    t->ctx = ctx;
    t->kernel = kernel;
    t->solver = solver;
    t->n_src = n_src;
    t->n_tgt = n_tgt;
    t->scalar = scalar;
    t->order = order;
    t->learned = solver.order_policy == LPM_ORDER_LEARNED;
    // the selector picks orders up to kMlpDirectClass (11); the fixed order is its fallback
    t->pm = t->learned ? std::max(kMlpDirectClass, order) : order;
    if (t->learned && solver.tolerance > 0.0) t->eps = solver.tolerance;
    // FP32 far field by default: its rounding stays ~1e-7 relative, below the truncation error of the
    // orders used; LPM_PREC_F64 evaluates every far expansion in FP64
    t->f64_from = solver.precision == LPM_PREC_F64 ? 1 : kPMax + 1;
    // about 4.7 * 4^L cells of level L meet the unit sphere (Biot-Savart); volume data (Poisson) fill up
    // to 8^L.  L is the level whose cells hold ~kBatch targets.  On the sphere batches are cut at the cells
    // of the next coarser level, so that the thinly populated cells the sphere only grazes merge with their
    // Morton neighbours and batches run fuller (measured: ~20% less far + near time at 2M targets).  In a
    // volume every cell is full, and a 128-target chunk of a coarser cell can straddle a Morton jump (two
    // distant sub-cells: a large batch radius and many more near pairs), so batches are cut at level L there
    // (1M points in [-1, 1]^3: 5.73 ms per evaluation against 6.91 ms at L - 1, 8.63e9 -> 5.03e9 near pairs);
    // the capacity is sized for one level finer than the default, the finest allowed.
    {
        const double grow = scalar ? 8.0 : 4.0, occ = scalar ? 1.0 : 4.7;
        int L = 1;
        while (L < kTreeDepth && occ * std::pow(grow, L + 1) * kBatch <= 1.5 * (double)n_tgt) ++L;
        t->batch_level = scalar ? L : std::max(1, L - 1);
        t->batch_level_max = scalar ? L + 1 : L;
        const int Lc = t->batch_level_max;
        const double cells_at_l = scalar ? std::pow(8.0, Lc) : 8.0 * std::pow(4.0, Lc);
        const int64_t cells = std::min<int64_t>(std::max<int64_t>(n_tgt, 1), (int64_t)cells_at_l + 64);
        t->n_batches = (n_tgt + kBatch - 1) / kBatch + cells;
    }
    if (sakajo > 0) {
        // SakajoTree: root Box3d(radius) padded by 1e-5 (src/LpmSakajo2009.cpp:25-39), 3L axis-cycling bisections
        rc = octree_alloc(t->st, std::max<int64_t>(n_src, 1), 0, 3 * sakajo, 1, kernel.radius);
        t->root_maxr = kernel.radius;
    } else {
        rc = octree_alloc(t->st, std::max<int64_t>(n_src, 1), solver.max_per_leaf, kTreeDepth);
    }
    if (rc) {
        delete t;
        return rc;
    }
    const size_t nn = (size_t)t->st.node_cap;
    std::vector<int4> ent, mono;  // mono in the packed moment order (mono_index)
    canonical_entries(t->pm, ent);
    for (int a = 0; a <= t->pm; ++a)
        for (int b = 0; a + b <= t->pm; ++b)
            for (int c = 0; a + b + c <= t->pm; ++c) mono.push_back(make_int4(a, b, c, 0));
    std::vector<int4> units;  // leaf moment units: runs of kP2mRun monomials along c
    for (int a = 0; a <= t->pm; ++a)
        for (int b = 0; a + b <= t->pm; ++b)
            for (int c = 0; a + b + c <= t->pm; c += kP2mRun) units.push_back(make_int4(a, b, c, 0));
    t->n_ent = (int)ent.size();
    t->n_mono = (int)mono.size();
    t->n_units = (int)units.size();
    // gather tables: for order P, the canonical index of each entry of the order-P Horner sequence
    std::vector<int32_t> gtab;
    for (int P = 1; P <= kPMax; ++P) {
        t->ct.table_off[P] = (int32_t)gtab.size();
        if (P > t->pm) continue;
        std::vector<int4> eP;
        canonical_entries(P, eP);
        for (const int4& e : eP) {
            int idx = -1;
            for (int i = 0; i < (int)ent.size(); ++i)
                if (ent[i].x == e.x && ent[i].y == e.y && ent[i].z == e.z && ent[i].w == e.w) {
                    idx = i;
                    break;
                }
            gtab.push_back(idx);
        }
    }
    t->ct.table_off[kPMax + 1] = (int32_t)gtab.size();
    // a cluster is cheaper to sum directly when its far-field work per target (8 flops per coefficient
    // plus ~40 of setup, at FP64 or FP32 rate) exceeds ~17 flops per direct pair at the FP32 rate
    for (int P = 0; P <= kPMax; ++P)
        t->ct.direct_below[P] = direct_cutoff(P, t->f64_from, t->scalar);
    cudaError_t e = cudaSuccess;
    auto A = [&](cudaError_t r) {
        if (e == cudaSuccess) e = r;
    };
    const size_t ns = (size_t)std::max<int64_t>(n_src, 1), ntg = (size_t)std::max<int64_t>(n_tgt, 1);
    A(talloc(t, &t->tkeys, ntg));
    A(talloc(t, &t->tperm, ntg));
    A(talloc(t, &t->ttmpk, ntg));
    A(talloc(t, &t->ttmpv, ntg));
    A(talloc(t, &t->tcount, 4));
    A(talloc(t, &t->tgt_sorted, ntg));
    A(talloc(t, &t->batch_ctr, (size_t)t->n_batches));
    A(talloc(t, &t->bflag, ntg + 1));
    A(talloc(t, &t->batch_first, (size_t)t->n_batches + 1));
    A(talloc(t, &t->src_sorted, ns));
    A(talloc(t, &t->src32, ns));
    A(talloc(t, &t->node_ctr, nn));
    A(talloc(t, &t->node_wabs, nn));
    // moments, coefficients and features (~40 KB per node at order 11) are sized for a realistic node
    // count, not the octree's worst case, and grown by uncaptured evaluations (heavy_alloc)
    t->heavy_cap = (int)std::min<int64_t>((int64_t)nn, sakajo > 0 ? 2 * std::max<int64_t>(n_src, 1) + 1024
                                                                   : 6 * (std::max<int64_t>(n_src, 1) /
                                                                          solver.max_per_leaf) + 1024);
    const size_t nh = (size_t)t->heavy_cap;
    A(talloc(t, &t->node_mom, nh * mono_count(t->pm)));
    if (scalar) {
        t->a_stride = (t->n_ent + 3) & ~3;  // 16-byte aligned rows in FP32 and FP64
        A(talloc(t, &t->A64, nh * t->a_stride));
        A(talloc(t, &t->A32, nh * t->a_stride));
    } else {
        A(talloc(t, &t->B64, nh * t->n_ent));
        A(talloc(t, &t->B32, nh * t->n_ent));
    }
    A(talloc(t, &t->ent, ent.size()));
    A(talloc(t, &t->mono, mono.size()));
    A(talloc(t, &t->p2m_units, units.size()));
    A(talloc(t, &t->m2m_pending, nn));
    A(talloc(t, &t->gtab, gtab.size()));
    const size_t far_rows = (size_t)(kPMax + 1) * ((size_t)t->n_batches + 1);  // order-bucketed rows
    A(talloc(t, &t->far_cnt, far_rows));
    A(talloc(t, &t->near_cnt, (size_t)t->n_batches + 1));
    A(talloc(t, &t->far_off, far_rows));
    A(talloc(t, &t->near_off, (size_t)t->n_batches + 1));
    A(talloc(t, &t->flags, 8));
    A(talloc(t, &t->root_r, 1));
    A(talloc(t, &t->near_work, (size_t)t->n_batches + 1));
    A(talloc(t, &t->far_work, (size_t)t->n_batches + 1));
    A(talloc(t, &t->sched_order, (size_t)t->n_batches + 1));
    A(talloc(t, &t->far_order, (size_t)t->n_batches + 1));
    A(talloc(t, &t->sched_aux, kAuxInts));
    A(talloc(t, &t->pair_counts, 3));
    A(talloc(t, &t->V, 3 * ntg));
    A(talloc(t, &t->W, scalar ? ntg : 1));
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&t->side, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&t->ev_fork, cudaEventDisableTiming);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&t->ev_join, cudaEventDisableTiming);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&t->ev_tfork, cudaEventDisableTiming);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&t->ev_tjoin, cudaEventDisableTiming);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&t->ev_cfork, cudaEventDisableTiming);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&t->ev_cjoin, cudaEventDisableTiming);
    if (t->learned) {
        A(talloc(t, &t->node_feat, nh * kMlpIn));
        A(talloc(t, &t->mlp_w, kMlpParams));
        A(talloc(t, &t->mlp_norm, 2 * kMlpIn));
        A(talloc(t, &t->decisions, (size_t)t->n_batches * kDecisionCap));
    }
    if (e == cudaSuccess) e = cudaMemcpy(t->ent, ent.data(), ent.size() * sizeof(int4), cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(t->mono, mono.data(), mono.size() * sizeof(int4), cudaMemcpyHostToDevice);
    if (e == cudaSuccess)
        e = cudaMemcpy(t->p2m_units, units.data(), units.size() * sizeof(int4), cudaMemcpyHostToDevice);
    if (e == cudaSuccess && !gtab.empty())
        e = cudaMemcpy(t->gtab, gtab.data(), gtab.size() * sizeof(int32_t), cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemset(t->node_mom, 0, nh * mono_count(t->pm) * sizeof(double));
    // the count arrays carry one extra zero entry so that their exclusive scans also yield the totals
    if (e == cudaSuccess) e = cudaMemset(t->far_cnt, 0, far_rows * sizeof(int32_t));
    if (e == cudaSuccess) e = cudaMemset(t->near_cnt, 0, ((size_t)t->n_batches + 1) * sizeof(int32_t));
    if (e != cudaSuccess) {
        tree_solver_destroy(t);
        return cuda_status(e, "tree solver allocation");
    }
    {
        cudaError_t ea = far_smem_attributes();
        // M2M stages two 8-child copies of the moments: opt in for the largest order any solver may use
        const int mono_max = (kPMax + 1) * (kPMax + 2) * (kPMax + 3) / 6;
        if (ea == cudaSuccess)
            ea = cudaFuncSetAttribute(m2m_upward_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      (int)(16 * mono_max * sizeof(double)));
        if (ea != cudaSuccess) {
            tree_solver_destroy(t);
            return cuda_status(ea, "cudaFuncSetAttribute (far_kernel)");
        }
        rc = near_shape(t, t->near_targets, t->near_tile, t->near_split);
        if (rc) {
            tree_solver_destroy(t);
            return rc;
        }
        int per_sm = 0;
        for (int P = 1; P <= kPMax && ea == cudaSuccess; ++P)
            for (int f64 = 0; f64 < 2 && ea == cudaSuccess; ++f64) {
                size_t smem = 0;
                int threads = 0;
                per_sm = 0;
                if (scalar) {
                    FarScalarFn fs = far_scalar_select(P, f64 != 0, &smem, &threads);
                    ea = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fs, threads, smem);
                } else {
                    FarKernelFn fn = far_kernel_select(P, f64 != 0, &smem, &threads);
                    ea = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fn, threads, smem);
                }
                t->far_blocks[P][f64] = (int)std::max<int64_t>(
                    1, std::min<int64_t>(t->n_batches, (int64_t)std::max(per_sm, 1) * ctx->num_sms));
            }
        for (int part = 1; part <= 2 && ea == cudaSuccess && !scalar; ++part) {
            size_t smem = 0;
            int threads = 0;
            per_sm = 0;
            FarKernelFn fn = far_split_select(part, &smem, &threads);
            ea = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fn, threads, smem);
            t->far_split_blocks[part - 1] = (int)std::max<int64_t>(
                1, std::min<int64_t>(t->n_batches, (int64_t)std::max(per_sm, 1) * ctx->num_sms));
        }
        if (ea == cudaSuccess && !scalar) {
            per_sm = 0;
            ea = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, far_low2_kernel, kFar2Threads, far_low_smem());
            t->far_low_blocks = (int)std::max<int64_t>(
                1, std::min<int64_t>(t->n_batches, (int64_t)std::max(per_sm, 1) * ctx->num_sms));
        }
        if (ea != cudaSuccess) {
            tree_solver_destroy(t);
            return cuda_status(ea, "cudaOccupancyMaxActiveBlocksPerMultiprocessor (far kernels)");
        }
    }
    rc = alloc_lists(t, std::max<int64_t>(t->n_batches * 256, 1024), std::max<int64_t>(t->n_batches * 64, 1024));
    if (rc) {
        tree_solver_destroy(t);
        return rc;
    }
    *out = t;
    return LPM_OK;
}

void tree_solver_destroy(TreeSolver* t) {
    if (!t) return;
    if (t->ev_fork) cudaEventDestroy(t->ev_fork);
    if (t->ev_join) cudaEventDestroy(t->ev_join);
    if (t->ev_tfork) cudaEventDestroy(t->ev_tfork);
    if (t->ev_tjoin) cudaEventDestroy(t->ev_tjoin);
    if (t->ev_cfork) cudaEventDestroy(t->ev_cfork);
    if (t->ev_cjoin) cudaEventDestroy(t->ev_cjoin);
    if (t->side) cudaStreamDestroy(t->side);
    octree_free(t->st);
    for (void* p : t->allocs) cudaFree(p);
    delete t;
}

static int build_lists(TreeSolver* t, bool can_sync) {
    lpm_ctx* ctx = t->ctx;
    TraverseArgs A{};
    A.t = t->st;
    A.node_ctr = t->node_ctr;
    A.batch_ctr = t->batch_ctr;
    A.batch_first = t->batch_first;
    A.nbat = t->tcount + 1;
    A.n_batches = t->n_batches;
    A.theta = t->solver.theta;
    A.order = t->order;
    A.direct_below = t->ct.direct_below[t->order];
    A.far_cnt = t->far_cnt;
    A.nb1 = t->n_batches + 1;
    A.near_cnt = t->near_cnt;
    A.far_off = t->far_off;
    A.near_off = t->near_off;
    A.flags = t->flags;
    A.pair_counts = t->pair_counts;
    A.fill = 0;
    A.learned = (t->learned && t->mlp_loaded) ? 1 : 0;
    A.max_order = std::min(t->pm, kMlpDirectClass);
    A.order_bias = t->order_bias;
    A.eps = t->eps;
    A.ct = t->ct;
    A.node_feat = t->node_feat;
    A.node_wabs = t->node_wabs;
    A.mlp_w = t->mlp_w;
    A.mlp_norm = t->mlp_norm;
    A.decisions = t->decisions;
    A.heavy_cap = t->heavy_cap;
    A.near_work = t->near_work;
    A.far_work = t->far_work;
    LPM_CUDA_TRY(cudaMemsetAsync(t->pair_counts, 0, 3 * sizeof(unsigned long long), ctx->stream));
    const unsigned g = grid_for(t->n_batches, 4);
    LPM_LAUNCH(ctx, "traverse_kernel", traverse_kernel, g, 128, 0, A);
    int rc = scan_exclusive_i32(ctx, t->far_cnt, t->far_off, (int64_t)(kPMax + 1) * (t->n_batches + 1), t->flags + 2);
    if (rc) return rc;
    rc = scan_exclusive_i32(ctx, t->near_cnt, t->near_off, t->n_batches + 1, t->flags + 3);
    if (rc) return rc;
    if (can_sync) {
        int32_t tot[2];
        LPM_CUDA_TRY(cudaMemcpyAsync(tot, t->flags + 2, sizeof(tot), cudaMemcpyDeviceToHost, ctx->stream));
        LPM_CUDA_TRY(cudaStreamSynchronize(ctx->stream));
        if (tot[0] > t->far_cap || tot[1] > t->near_cap) {
            rc = alloc_lists(t, std::max<int64_t>(t->far_cap, (int64_t)(tot[0] * 1.5) + 1024),
                             std::max<int64_t>(t->near_cap, (int64_t)(tot[1] * 1.5) + 1024));
            if (rc) return rc;
        }
    }
    A.fill = 1;
    A.far_list = t->far_list;
    A.near_list = t->near_list;
    A.far_cap = t->far_cap;
    A.near_cap = t->near_cap;
    LPM_LAUNCH(ctx, "traverse_kernel", traverse_kernel, g, 128, 0, A);
    return LPM_OK;
}

// The far-field orders of an evaluation: the fixed order, or the selector's orders 1..11.
static void far_order_range(const TreeSolver* t, int* p_lo, int* p_hi) {
    const bool sel = t->learned && t->mlp_loaded;
    *p_lo = sel ? 1 : t->order;
    *p_hi = sel ? std::min(t->pm, kMlpDirectClass) : t->order;
}

// Everything of an evaluation before its far and near fields: root box, target batches, source octree, moments,
// coefficients, interaction lists, V cleared and, with `sched`, the batch schedules of the solver's own
// persistent far and near launches.  *pending is false when the evaluation is complete already (no targets or
// no sources).
static int tree_prepare(TreeSolver* t, const double4* src, int64_t n_src, const double4* X, int64_t n_tgt,
                        double* U, bool sched, bool* pending) {
    lpm_ctx* ctx = t->ctx;
    *pending = false;
    if (n_src != t->n_src || n_tgt != t->n_tgt) {
        set_error("tree_velocity: sizes differ from the solver's");
        return LPM_ERR_ARG;
    }
    cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
    LPM_CUDA_TRY(cudaStreamIsCapturing(ctx->stream, &cap));
    const bool can_sync = cap == cudaStreamCaptureStatusNone;
    if (n_tgt == 0) return LPM_OK;
    if (n_src == 0) {
        LPM_CUDA_TRY(cudaMemsetAsync(U, 0, (t->scalar ? 1 : 3) * (size_t)n_tgt * sizeof(double), ctx->stream));
        return LPM_OK;
    }
    LPM_CUDA_TRY(cudaMemsetAsync(t->flags, 0, 8 * sizeof(int32_t), ctx->stream));
    RootBox rb;
    int rc = LPM_OK;
    if (!t->scalar && t->root_maxr > 0.0) {
        for (int a = 0; a < 3; ++a) {
            rb.lo[a] = -t->root_maxr - 1e-5;
            rb.hi[a] = t->root_maxr + 1e-5;
        }
    } else {
        rb.r_dev = t->root_r;
        rb.mode = t->scalar ? kRootMaxNorm : kRootEuclid;
        if (!t->scalar && t->root_first < n_tgt)
            rc = root_extent(ctx, X, t->root_first, n_tgt, kRootEuclid, t->root_r);
        else
            rc = root_extent(ctx, src, 0, n_src, rb.mode, t->root_r);
        if (rc) return rc;
    }
    // targets in Morton order, cut into compact batches of at most kBatch.  Independent of the source tree until
    // the traversal, so (profiling off) it runs on the solver's side stream while the source octree and its
    // moments are built on the context's stream: both are chains of short latency-bound launches.  Its sort and
    // scan use their own scratch slots.
    const unsigned gt = (unsigned)std::max<int64_t>(1, std::min<int64_t>(grid_for(n_tgt + 1, 256), 8 * ctx->num_sms));
    auto target_batches = [&]() -> int {
        LPM_CUDA_TRY(cudaMemsetAsync(t->tcount, 0, 4 * sizeof(int32_t), ctx->stream));
        int r = morton_keys(ctx, X, n_tgt, rb, t->tkeys, t->tperm, t->tcount);
        if (r) return r;
        r = radix_sort_u64(ctx, t->tkeys, t->tperm, t->ttmpk, t->ttmpv, n_tgt, 32, kSlotSideCounts, kSlotSideSums);
        if (r) return r;
        LPM_CUDA_TRY(cudaMemsetAsync(t->bflag + n_tgt, 0, sizeof(int32_t), ctx->stream));
        LPM_LAUNCH(ctx, "batch_flags_kernel", batch_flags_kernel, gt, 256, 0, t->tkeys, n_tgt,
                   3 * (kKeyLevels - t->batch_level), t->bflag);
        r = scan_exclusive_i32(ctx, t->bflag, t->bflag, n_tgt + 1, nullptr, kSlotSideSums);
        if (r) return r;
        LPM_LAUNCH(ctx, "batch_first_kernel", batch_first_kernel, gt, 256, 0, t->bflag, n_tgt, t->batch_first,
                   t->tcount + 1, t->n_batches);
        LPM_LAUNCH(ctx, "batch_kernel", batch_kernel, (unsigned)t->n_batches, kBatch, 0, X, t->tperm,
                   t->batch_first, t->tcount + 1, t->tgt_sorted, t->batch_ctr);
        return LPM_OK;
    };
    const bool tside = !ctx->profiling;
    if (tside) {
        LPM_CUDA_TRY(cudaEventRecord(t->ev_tfork, ctx->stream));
        LPM_CUDA_TRY(cudaStreamWaitEvent(t->side, t->ev_tfork, 0));
        cudaStream_t main_stream = ctx->stream;
        ctx->stream = t->side;
        rc = target_batches();
        ctx->stream = main_stream;
        if (rc) return rc;
        LPM_CUDA_TRY(cudaEventRecord(t->ev_tjoin, t->side));
    }
    rc = octree_build(ctx, t->st, src, n_src, rb);
    if (rc) return rc;
    if (can_sync) {  // grow the per-node arrays to this tree (a captured replay can only flag an overflow)
        int32_t nodes = 0;
        LPM_CUDA_TRY(cudaMemcpyAsync(&nodes, t->st.counters + 1, sizeof(int32_t), cudaMemcpyDeviceToHost,
                                     ctx->stream));
        LPM_CUDA_TRY(cudaStreamSynchronize(ctx->stream));
        if (nodes > t->heavy_cap) {
            rc = heavy_alloc(t, nodes);
            if (rc) return rc;
        }
    }
    const unsigned gs = (unsigned)std::max<int64_t>(1, std::min<int64_t>(grid_for(n_src, 256), 8 * ctx->num_sms));
    LPM_LAUNCH(ctx, "gather_sources_kernel", gather_sources_kernel, gs, 256, 0, src, t->st.perm, t->st.counters,
               t->src_sorted);
    const unsigned gl = (unsigned)std::max<int64_t>(1, std::min<int64_t>(t->st.node_cap, 16 * ctx->num_sms));
    LPM_LAUNCH(ctx, "leaf_p2m_kernel", leaf_p2m_kernel, gl, kP2mThreads, 0, t->st, t->src_sorted, t->pm, t->p2m_units,
               t->n_units,
               t->node_ctr, t->node_wabs, t->node_mom, t->src32, t->scalar ? 1.0 : 2.0, t->heavy_cap);
    LPM_LAUNCH(ctx, "m2m_pending_kernel", m2m_pending_kernel, gl, 128, 0, t->st, t->m2m_pending);
    LPM_LAUNCH(ctx, "m2m_upward_kernel", m2m_upward_kernel, gl, kM2mThreads, (size_t)16 * t->n_mono * sizeof(double), t->st,
               t->pm, t->mono, t->n_mono, t->node_ctr, t->node_wabs, t->node_mom, t->heavy_cap, t->m2m_pending);
    // far-field coefficients: needed only by the far kernels, so (profiling off) on the side stream during the
    // node features and the traversal
    auto coefficients = [&]() -> int {
        if (t->scalar)
            LPM_LAUNCH(ctx, "coeff_kernel", coeff_scalar_kernel, gl, 128, 0, t->st, t->pm, t->ent, t->n_ent,
                       t->a_stride, t->node_mom, t->A64, t->A32, t->heavy_cap);
        else
            LPM_LAUNCH(ctx, "coeff_kernel", coeff_kernel, gl, 128, 0, t->st, t->pm, t->ent, t->n_ent, t->node_mom,
                       t->B64, t->B32, t->heavy_cap);
        return LPM_OK;
    };
    if (tside) {
        LPM_CUDA_TRY(cudaEventRecord(t->ev_cfork, ctx->stream));
        LPM_CUDA_TRY(cudaStreamWaitEvent(t->side, t->ev_cfork, 0));
        cudaStream_t main_stream = ctx->stream;
        ctx->stream = t->side;
        rc = coefficients();
        ctx->stream = main_stream;
        if (rc) return rc;
        LPM_CUDA_TRY(cudaEventRecord(t->ev_cjoin, t->side));
    } else {
        rc = coefficients();
        if (rc) return rc;
    }
    if (t->learned)
        LPM_LAUNCH(ctx, "node_feature_kernel", node_feature_kernel, gl, 128, 0, t->st, t->pm, t->node_ctr,
                   t->node_wabs, t->node_mom, t->node_feat, t->heavy_cap);
    if (tside) {  // the target batches were formed on the side stream
        LPM_CUDA_TRY(cudaStreamWaitEvent(ctx->stream, t->ev_tjoin, 0));
    } else {
        rc = target_batches();
        if (rc) return rc;
    }
    rc = build_lists(t, can_sync);
    if (rc) return rc;
    if (tside) LPM_CUDA_TRY(cudaStreamWaitEvent(ctx->stream, t->ev_cjoin, 0));  // the coefficients
    // far field: one launch per order present (only the fixed order, or the selector's orders 1..11),
    // each adding its bucket's contributions to V
    LPM_CUDA_TRY(cudaMemsetAsync(t->V, 0, 3 * (size_t)n_tgt * sizeof(double), ctx->stream));
    *pending = true;
    if (!sched) return LPM_OK;
    // batch schedules: far and near work of every batch (from the traversal's count pass), bucketed in
    // decreasing order; zeroed buckets, cursors and tickets first
    LPM_CUDA_TRY(cudaMemsetAsync(t->sched_aux, 0, kAuxInts * sizeof(int32_t), ctx->stream));
    const unsigned gsch = (unsigned)std::max<int64_t>(1, std::min<int64_t>(grid_for(t->n_batches, 256),
                                                                            2 * ctx->num_sms));
    LPM_LAUNCH(ctx, "sched_hist_kernel", sched_hist_kernel, gsch, 256, 0, t->far_work, t->tcount + 1,
               t->sched_aux + kAuxFarHist);
    LPM_LAUNCH(ctx, "sched_scatter_kernel", sched_scatter_kernel, gsch, 256, 0, t->far_work, t->tcount + 1,
               t->sched_aux + kAuxFarHist, t->sched_aux + kAuxFarCur, t->far_order);
    LPM_LAUNCH(ctx, "sched_hist_kernel", sched_hist_kernel, gsch, 256, 0, t->near_work, t->tcount + 1,
               t->sched_aux + kAuxNearHist);
    LPM_LAUNCH(ctx, "sched_scatter_kernel", sched_scatter_kernel, gsch, 256, 0, t->near_work, t->tcount + 1,
               t->sched_aux + kAuxNearHist, t->sched_aux + kAuxNearCur, t->sched_order);
    return LPM_OK;
}

// The far kernels' arguments for order P of t's current evaluation (schedule: t's own).
static FarArgs far_args(const TreeSolver* t, int P) {
    const int64_t nb1 = t->n_batches + 1;
    FarArgs F{};
    F.tgt_sorted = t->tgt_sorted;
    F.n_tgt = t->n_tgt;
    F.batch_first = t->batch_first;
    F.nbat = t->tcount + 1;
    F.far_off = t->far_off + (size_t)P * nb1;
    F.far_cnt = t->far_cnt + (size_t)P * nb1;
    F.far_list = t->far_list;
    F.far_cap = t->far_cap;
    F.node_ctr = t->node_ctr;
    F.B64 = t->B64;
    F.B32 = t->B32;
    F.n_ent = t->n_ent;
    F.gtab = t->gtab + t->ct.table_off[P];
    F.V = t->V;
    F.order = t->far_order;
    F.ticket = t->sched_aux + kAuxFarTicket + P;
    return F;
}

// The near kernel's arguments for t's current evaluation, writing the result to U (schedule: t's own).
static NearArgs near_args(const TreeSolver* t, double* U) {
    NearArgs N{};
    N.t = t->st;
    N.tgt_sorted = t->tgt_sorted;
    N.n_tgt = t->n_tgt;
    N.batch_first = t->batch_first;
    N.nbat = t->tcount + 1;
    N.near_off = t->near_off;
    N.near_cnt = t->near_cnt;
    N.near_list = t->near_list;
    N.near_cap = t->near_cap;
    N.src32 = t->src32;
    N.W = t->W;
    N.tperm = t->tperm;
    N.V = t->V;
    N.mult = -1.0 / (4.0 * kPi * t->kernel.radius);
    N.U = U;
    N.order = t->sched_order;
    N.ticket = t->sched_aux + kAuxNearTicket;
    return N;
}

// Order P's far-field launch(es) of t on its context's stream, on the schedule tree_prepare made.
static int tree_far_order(TreeSolver* t, int P) {
    lpm_ctx* ctx = t->ctx;
    FarArgs F = far_args(t, P);
    size_t smem = 0;
    const bool f64 = P >= t->f64_from;
    const unsigned grid = (unsigned)t->far_blocks[P][f64 ? 1 : 0];
    if (t->scalar) {
        F.B64 = (const double4*)t->A64;
        F.B32 = (const float4*)t->A32;
        int threads = 0;
        FarScalarFn fs = far_scalar_select(P, f64, &smem, &threads);
        LPM_LAUNCH(ctx, "far_kernel", fs, grid, threads, smem, F, t->a_stride);
    } else if (P == kFarSplitOrder && !f64) {  // two launches, each on its own ticket
        for (int part = 1; part <= 2; ++part) {
            int threads = 0;
            FarKernelFn fn = far_split_select(part, &smem, &threads);
            F.gtab = t->gtab + t->ct.table_off[P] + (part == 2 ? part_entries(P, 1) : 0);
            F.ticket = t->sched_aux + kAuxFarTicket + (part == 2 ? kPMax + 1 : P);
            LPM_LAUNCH(ctx, "far_kernel", fn, (unsigned)t->far_split_blocks[part - 1], threads, smem, F);
        }
    } else {
        int threads = 0;
        FarKernelFn fn = far_kernel_select(P, f64, &smem, &threads);
        LPM_LAUNCH(ctx, "far_kernel", fn, grid, threads, smem, F);
    }
    return LPM_OK;
}

int tree_velocity(TreeSolver* t, const double4* src, int64_t n_src, const double4* X, int64_t n_tgt, double* U) {
    lpm_ctx* ctx = t->ctx;
    bool pending = false;
    int rc = tree_prepare(t, src, n_src, X, n_tgt, U, true, &pending);
    if (rc || !pending) return rc;
    cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
    LPM_CUDA_TRY(cudaStreamIsCapturing(ctx->stream, &cap));
    const bool can_sync = cap == cudaStreamCaptureStatusNone;
    const unsigned gt = (unsigned)std::max<int64_t>(1, std::min<int64_t>(grid_for(n_tgt + 1, 256), 8 * ctx->num_sms));
    // near field: batches by decreasing near work, taken by a persistent grid.  Biot-Savart: after the far
    // field on the context's stream, writing u = mult (V - x cross D).  Scalar kernel: it writes W only and runs
    // on the solver's side stream beside the far-field launch, filling its tail (1M Poisson points: 7.37 ->
    // 7.14 ms per evaluation; on the sphere the same overlap measured no gain), then a combine kernel forms
    // u; with per-kernel profiling on it runs after the far field on the context's stream, so that every kernel
    // is timed alone.
    auto launch_near = [&]() -> int {
        const NearArgs N = near_args(t, U);
        int threads = 0;
        NearFn fn = near_select(t->scalar, t->near_targets, t->near_tile, t->near_split, &threads);
        LPM_LAUNCH(ctx, "near_kernel", fn, (unsigned)t->near_blocks, threads, 0, N);
        return LPM_OK;
    };
    const bool overlap = t->scalar && !ctx->profiling;
    if (overlap) LPM_CUDA_TRY(cudaEventRecord(t->ev_fork, ctx->stream));
    int p_lo = 0, p_hi = -1;
    far_order_range(t, &p_lo, &p_hi);
    const int low_hi = std::min(p_hi, kFarLowMax);
    if (!t->scalar && low_hi > p_lo && low_hi < t->f64_from) {  // FP32 orders p_lo..low_hi in one launch
        FarLowArgs LA{};
        for (int P = p_lo; P <= low_hi; ++P) LA.a[P - 1] = far_args(t, P);
        LPM_LAUNCH(ctx, "far_kernel", far_low2_kernel, (unsigned)t->far_low_blocks, kFar2Threads, far_low_smem(), LA,
                   t->tcount + 1, t->far_order, t->sched_aux + kAuxFarTicket + p_lo);
        p_lo = low_hi + 1;
    }
    for (int P = p_lo; P <= p_hi; ++P) {
        rc = tree_far_order(t, P);
        if (rc) return rc;
    }
    if (overlap) {  // enqueued after the far launches: the near blocks fill the SMs as far blocks retire
        LPM_CUDA_TRY(cudaStreamWaitEvent(t->side, t->ev_fork, 0));
        cudaStream_t main_stream = ctx->stream;
        ctx->stream = t->side;
        rc = launch_near();
        ctx->stream = main_stream;
        if (rc) return rc;
        LPM_CUDA_TRY(cudaEventRecord(t->ev_join, t->side));
        LPM_CUDA_TRY(cudaStreamWaitEvent(ctx->stream, t->ev_join, 0));
    } else {
        rc = launch_near();
        if (rc) return rc;
    }
    if (t->scalar)
        LPM_LAUNCH(ctx, "combine_kernel", far_near_combine_kernel, gt, 256, 0, t->V, t->W, t->tperm, n_tgt,
                   1.0 / (4.0 * kPi), U);
    if (can_sync) return tree_check(t);
    return LPM_OK;
}

// ---------------------------------------------------------------------------------- fused solvers (host)
struct TreeFused {
    lpm_ctx* ctx = nullptr;  // its stream carries the fused launches
    int n = 0;               // solvers bound
    int inst_cap = 0;
    int64_t item_cap = 0;
    std::vector<TreeSolver*> ts;
    FusedInst* inst = nullptr;   // device, n
    FarArgs* far_tab = nullptr;  // device, kFusedFarSlots x n (slot-major)
    NearArgs* near_tab = nullptr;  // device, kFusedNearGroups x n (group-major)
    int2* far_items = nullptr;
    int2* near_items = nullptr;
    int32_t* aux = nullptr;
    bool far_on[kFusedFarSlots] = {};
    std::vector<int4> groups;                 // near tile shapes present: (targets, tile, split, -)
    std::vector<std::pair<int, int>> single;  // (solver, order) far launches outside the fused kernels
    int64_t max_batches = 0;
};

// Whether every far order of t runs in the fused FP32 kernels (else t also keeps its own schedule for the
// orders that do not).
static bool fused_far_all(const TreeSolver* t) {
    int p_lo = 0, p_hi = -1;
    far_order_range(t, &p_lo, &p_hi);
    return !t->scalar && p_hi <= kFar2MaxOrder && p_hi < t->f64_from;
}

// Whether t takes part in fused launches: a Biot-Savart evaluation with sources and targets.
static bool fused_part(const TreeSolver* t) { return t && !t->scalar && t->n_src > 0 && t->n_tgt > 0; }

int tree_fused_create(lpm_ctx* ctx, TreeFused** out) {
    *out = nullptr;
    TreeFused* f = new (std::nothrow) TreeFused();
    if (!f) return LPM_ERR_OOM;
    f->ctx = ctx;
    *out = f;
    return LPM_OK;
}

static void fused_free(TreeFused* f) {
    cudaFree(f->inst);
    cudaFree(f->far_tab);
    cudaFree(f->near_tab);
    cudaFree(f->far_items);
    cudaFree(f->near_items);
    cudaFree(f->aux);
    f->inst = nullptr;
    f->far_tab = nullptr;
    f->near_tab = nullptr;
    f->far_items = f->near_items = nullptr;
    f->aux = nullptr;
    f->inst_cap = 0;
    f->item_cap = 0;
}

void tree_fused_destroy(TreeFused* f) {
    if (!f) return;
    fused_free(f);
    delete f;
}

int tree_fused_prepare(TreeSolver* t, const double4* src, const double4* X, double* U) {
    bool pending = false;
    return tree_prepare(t, src, t->n_src, X, t->n_tgt, U, !fused_far_all(t), &pending);
}

int tree_fused_bind(TreeFused* f, TreeSolver* const* ts, double* const* Us, int n) {
    if (n < 1 || n > 65535) {
        set_error("fused solvers: 1 to 65535 solvers");
        return LPM_ERR_ARG;
    }
    int64_t items = 0, max_nb = 0;
    for (int i = 0; i < n; ++i)
        if (fused_part(ts[i])) {
            items += ts[i]->n_batches;
            max_nb = std::max(max_nb, ts[i]->n_batches);
        }
    LPM_CUDA_TRY(cudaSetDevice(f->ctx->device));
    if (n > f->inst_cap || items > f->item_cap) {
        fused_free(f);
        const int cap = std::max(n, 1);
        const int64_t icap = std::max<int64_t>(items, 1);
        cudaError_t e = dev_alloc((void**)&f->inst, sizeof(FusedInst) * (size_t)cap);
        if (e == cudaSuccess) e = dev_alloc((void**)&f->far_tab, sizeof(FarArgs) * kFusedFarSlots * (size_t)cap);
        if (e == cudaSuccess) e = dev_alloc((void**)&f->near_tab, sizeof(NearArgs) * kFusedNearGroups * (size_t)cap);
        if (e == cudaSuccess) e = dev_alloc((void**)&f->far_items, sizeof(int2) * (size_t)icap);
        if (e == cudaSuccess) e = dev_alloc((void**)&f->near_items, sizeof(int2) * (size_t)icap);
        if (e == cudaSuccess) e = dev_alloc((void**)&f->aux, sizeof(int32_t) * kFzInts);
        if (e != cudaSuccess) {
            fused_free(f);
            return cuda_status(e, "cudaMalloc (fused solvers)");
        }
        f->inst_cap = cap;
        f->item_cap = icap;
    }
    std::vector<FusedInst> hinst((size_t)n, FusedInst{nullptr, nullptr, nullptr});
    std::vector<FarArgs> hfar((size_t)kFusedFarSlots * n, FarArgs{});
    std::vector<NearArgs> hnear((size_t)kFusedNearGroups * n, NearArgs{});
    f->ts.assign(ts, ts + n);
    f->n = n;
    f->groups.clear();
    f->single.clear();
    for (bool& on : f->far_on) on = false;
    for (int i = 0; i < n; ++i) {
        TreeSolver* t = ts[i];
        if (!fused_part(t)) continue;
        hinst[i] = FusedInst{t->far_work, t->near_work, t->tcount + 1};
        int p_lo = 0, p_hi = -1;
        far_order_range(t, &p_lo, &p_hi);
        for (int P = p_lo; P <= p_hi; ++P) {
            if (P > kFar2MaxOrder || P >= t->f64_from) {
                f->single.emplace_back(i, P);
                continue;
            }
            hfar[(size_t)P * n + i] = far_args(t, P);
            f->far_on[P] = true;
            if (P == kFarSplitOrder) {
                FarArgs F2 = far_args(t, P);
                F2.gtab += part_entries(P, 1);
                hfar[(size_t)(kPMax + 1) * n + i] = F2;
                f->far_on[kPMax + 1] = true;
            }
        }
        int g = 0;
        while (g < (int)f->groups.size() && !(f->groups[g].x == t->near_targets && f->groups[g].y == t->near_tile &&
                                                f->groups[g].z == t->near_split))
            ++g;
        if (g == (int)f->groups.size()) {
            if (g == kFusedNearGroups) {
                set_error("fused solvers: too many near tile shapes");
                return LPM_ERR_ARG;
            }
            f->groups.push_back(make_int4(t->near_targets, t->near_tile, t->near_split, 0));
        }
        hnear[(size_t)g * n + i] = near_args(t, Us[i]);
    }
    f->max_batches = max_nb;
    cudaStream_t s = f->ctx->stream;
    LPM_CUDA_TRY(cudaMemcpyAsync(f->inst, hinst.data(), sizeof(FusedInst) * hinst.size(), cudaMemcpyHostToDevice, s));
    LPM_CUDA_TRY(cudaMemcpyAsync(f->far_tab, hfar.data(), sizeof(FarArgs) * hfar.size(), cudaMemcpyHostToDevice, s));
    LPM_CUDA_TRY(cudaMemcpyAsync(f->near_tab, hnear.data(), sizeof(NearArgs) * hnear.size(), cudaMemcpyHostToDevice,
                                 s));
    LPM_CUDA_TRY(cudaStreamSynchronize(s));  // the host tables go out of scope
    return LPM_OK;
}

// Persistent grid of a fused kernel: its resident blocks on the whole device.
template <typename Fn>
static int fused_grid(lpm_ctx* ctx, Fn fn, int threads, size_t smem, unsigned* grid) {
    int per_sm = 0;
    LPM_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fn, threads, smem));
    *grid = (unsigned)(std::max(per_sm, 1) * ctx->num_sms);
    return LPM_OK;
}

int tree_fused_run(TreeFused* f) {
    lpm_ctx* ctx = f->ctx;
    const int n = f->n;
    if (n < 1) {
        set_error("fused solvers: nothing bound");
        return LPM_ERR_ARG;
    }
    LPM_CUDA_TRY(cudaMemsetAsync(f->aux, 0, kFzInts * sizeof(int32_t), ctx->stream));
    const dim3 gsch((unsigned)std::max<int64_t>(1, std::min<int64_t>(grid_for(f->max_batches, 256), 64)),
                    (unsigned)n);
    LPM_LAUNCH(ctx, "fused_hist_kernel", fused_hist_kernel, gsch, 256, 0, f->inst, f->aux);
    LPM_LAUNCH(ctx, "fused_scatter_kernel", fused_scatter_kernel, gsch, 256, 0, f->inst, f->aux, f->far_items,
               f->near_items);
    for (int P = 1; P <= kPMax; ++P) {
        for (int part = 1; part <= 2; ++part) {  // part 2: the second launch of kFarSplitOrder
            const int slot = part == 1 ? P : kPMax + 1;
            if (part == 2 && P != kFarSplitOrder) break;
            if (!f->far_on[slot]) continue;
            size_t smem = 0;
            int threads = 0;
            FarFusedFn fn = far_fused_select(P, P == kFarSplitOrder ? part : 0, &smem, &threads);
            if (!fn) {
                set_error("fused solvers: no fused far kernel of order %d", P);
                return LPM_ERR_ARG;
            }
            unsigned grid = 0;
            int rc = fused_grid(ctx, fn, threads, smem, &grid);
            if (rc) return rc;
            const FusedSched S{f->far_items, f->aux + kFzTotals, f->aux + kFzFarTicket + slot};
            LPM_LAUNCH(ctx, "far_kernel", fn, grid, threads, smem, f->far_tab + (size_t)slot * n, S);
        }
        for (const auto& sp : f->single) {  // orders outside the fused kernels: the solver's own launch
            if (sp.second != P) continue;
            TreeSolver* t = f->ts[sp.first];
            cudaStream_t own = t->ctx->stream;
            t->ctx->stream = ctx->stream;
            const int rc = tree_far_order(t, P);
            t->ctx->stream = own;
            if (rc) return rc;
        }
    }
    for (size_t g = 0; g < f->groups.size(); ++g) {
        int threads = 0;
        NearFusedFn fn = near_fused_select(f->groups[g].x, f->groups[g].y, f->groups[g].z, &threads);
        if (!fn) {
            set_error("fused solvers: no fused near kernel of this tile shape");
            return LPM_ERR_ARG;
        }
        unsigned grid = 0;
        int rc = fused_grid(ctx, fn, threads, 0, &grid);
        if (rc) return rc;
        const FusedSched S{f->near_items, f->aux + kFzTotals + 1, f->aux + kFzNearTicket + (int)g};
        LPM_LAUNCH(ctx, "near_kernel", fn, grid, threads, 0, f->near_tab + g * (size_t)n, S);
    }
    return LPM_OK;
}

int tree_check(TreeSolver* t) {
    if (t->n_src == 0 || t->n_tgt == 0) return LPM_OK;  // its evaluations build no tree and fill no lists
    int32_t f[8], c[8], tc[4];
    lpm_ctx* ctx = t->ctx;
    LPM_CUDA_TRY(cudaMemcpyAsync(f, t->flags, sizeof(f), cudaMemcpyDeviceToHost, ctx->stream));
    LPM_CUDA_TRY(cudaMemcpyAsync(c, t->st.counters, sizeof(c), cudaMemcpyDeviceToHost, ctx->stream));
    LPM_CUDA_TRY(cudaMemcpyAsync(tc, t->tcount, sizeof(tc), cudaMemcpyDeviceToHost, ctx->stream));
    LPM_CUDA_TRY(cudaStreamSynchronize(ctx->stream));
    if (f[0]) {
        set_error("tree solver: capacity exceeded in a captured evaluation (flags %d: 1 far list, 2 near list, "
                  "4 traversal stack, 16 node moments); run one uncaptured evaluation to regrow", f[0]);
        return LPM_ERR_CAPACITY;
    }
    if (tc[1] > t->n_batches) {
        set_error("tree solver: %d target batches exceed the capacity of %lld", tc[1], (long long)t->n_batches);
        return LPM_ERR_CAPACITY;
    }
    if (c[2] & 2) {
        set_error("tree solver: octree node capacity exhausted");
        return LPM_ERR_CAPACITY;
    }
    if (c[0] != t->n_src) {
        set_error("tree solver: %d of %lld sources lie outside the root box (non-finite coordinates, or sources "
                  "beyond the targets' maxR)", (int)(t->n_src - c[0]), (long long)t->n_src);
        return LPM_ERR_ARG;
    }
    return LPM_OK;
}

uint64_t tree_generation(const TreeSolver* t) { return t->generation; }

const Octree& tree_source_octree(const TreeSolver* t, int64_t* n_points) {
    *n_points = t->n_src;
    return t->st;
}

int tree_stats(TreeSolver* t, int64_t* out8) {
    if (t->n_src == 0 || t->n_tgt == 0) {  // no tree, no lists
        for (int k = 0; k < 10; ++k) out8[k] = 0;
        return LPM_OK;
    }
    int32_t f[8], c[8];
    unsigned long long pc[3];
    lpm_ctx* ctx = t->ctx;
    LPM_CUDA_TRY(cudaMemcpyAsync(pc, t->pair_counts, sizeof(pc), cudaMemcpyDeviceToHost, ctx->stream));
    LPM_CUDA_TRY(cudaMemcpyAsync(f, t->flags, sizeof(f), cudaMemcpyDeviceToHost, ctx->stream));
    LPM_CUDA_TRY(cudaMemcpyAsync(c, t->st.counters, sizeof(c), cudaMemcpyDeviceToHost, ctx->stream));
    LPM_CUDA_TRY(cudaStreamSynchronize(ctx->stream));
    out8[0] = c[1];   // nodes
    out8[1] = c[3];   // leaves
    out8[2] = c[4];   // depth
    out8[3] = f[2];   // far (batch, cluster) pairs
    out8[4] = f[3];   // near runs
    int32_t tc[4];
    LPM_CUDA_TRY(cudaMemcpy(tc, t->tcount, sizeof(tc), cudaMemcpyDeviceToHost));
    out8[5] = tc[1];  // target batches
    out8[6] = f[0];
    out8[7] = (int64_t)pc[0];  // far-field target-cluster evaluations
    out8[8] = (int64_t)pc[1];  // near-field target-source pairs
    out8[9] = (int64_t)pc[2];  // far coefficient evaluations: sum of E(P) over far evaluations
    return LPM_OK;
}

}  // namespace lpm

namespace lpm {

int tree_get_param(const TreeSolver* t, const char* name, double* value) {
    if (!name || !value) {
        set_error("tree_get_param: null argument");
        return LPM_ERR_ARG;
    }
    const std::string n(name);
    if (n == "theta") *value = t->solver.theta;
    else if (n == "eps") *value = t->eps;
    else if (n == "f64_from") *value = t->f64_from;
    else if (n == "order_bias") *value = t->order_bias;
    else if (n == "batch_level") *value = t->batch_level;
    else if (n == "batch_level_max") *value = t->batch_level_max;
    else if (n == "sakajo_depth") *value = t->solver.sakajo_depth;
    else if (n == "near_targets") *value = t->near_targets;
    else if (n == "near_tile") *value = t->near_tile;
    else if (n == "near_split") *value = t->near_split;
    else if (n == "root_maxr") *value = t->root_maxr;
    else if (n == "root_first") *value = (double)t->root_first;
    else if (n == "order") *value = t->order;
    else {
        set_error("tree_get_param: unknown parameter %s", name);
        return LPM_ERR_ARG;
    }
    return LPM_OK;
}

int tree_set_param(TreeSolver* t, const char* name, double value) {
    if (!name) {
        set_error("tree_set_param: null name");
        return LPM_ERR_ARG;
    }
    const std::string n(name);
    if (n == "theta" && value > 0.0 && value < 1.0) {
        t->solver.theta = value;
    } else if (n == "eps" && value > 0.0) {
        t->eps = value;
    } else if (n == "order_bias" && value >= 0.0 && value <= 3.0 && value == std::floor(value)) {
        if (!t->learned) {
            set_error("tree_set_param: order_bias applies to LPM_ORDER_LEARNED solvers only");
            return LPM_ERR_ARG;
        }
        t->order_bias = (int)value;
    } else if (n == "near_targets" && (value == 2.0 || value == 4.0)) {
        return near_shape(t, (int)value, t->near_tile, t->near_split);
    } else if (n == "near_tile" && (value == 256.0 || value == 512.0 || value == 1024.0)) {
        return near_shape(t, t->near_targets, (int)value, t->near_split);
    } else if (n == "near_split" && (value == 1.0 || value == 2.0)) {
        return near_shape(t, t->near_targets, t->near_tile, (int)value);
    } else if (n == "root_maxr" && value >= 0.0 && std::isfinite(value)) {
        t->root_maxr = value;
    } else if (n == "root_first" && value >= 0.0 && value <= (double)t->n_tgt && value == std::floor(value)) {
        t->root_first = (int64_t)value;
    } else if (n == "batch_level" && value >= 1.0 && value <= t->batch_level_max && value == std::floor(value)) {
        t->batch_level = (int)value;
    } else if (n == "f64_from" && value >= 1.0 && value <= kPMax + 1 && value == std::floor(value)) {
        t->f64_from = (int)value;
        for (int P = 1; P <= kPMax; ++P) t->ct.direct_below[P] = direct_cutoff(P, t->f64_from, t->scalar);
    } else {
        set_error("tree_set_param: unknown parameter or value out of range: %s = %g", name, value);
        return LPM_ERR_ARG;
    }
    return LPM_OK;
}

}  // namespace lpm

namespace lpm {

int tree_set_mlp(TreeSolver* t, const float* params_host) {
    if (!t->learned) {
        set_error("tree solver: the order selector applies to LPM_ORDER_LEARNED solvers only");
        return LPM_ERR_ARG;
    }
    if (!params_host) {
        t->mlp_loaded = false;  // back to the fixed-order fallback
        return LPM_OK;
    }
    int rc = mlp_upload_bf16(t->ctx, params_host, t->mlp_w, t->mlp_norm);
    if (rc) return rc;
    t->mlp_loaded = true;
    return LPM_OK;
}

namespace {
struct TmpBuf {
    void* p = nullptr;
    ~TmpBuf() {
        if (p) cudaFree(p);
    }
};
}  // namespace

// One evaluation with every accepted cluster listed as a far entry (fixed-order lists, no cost cutoff),
// then the sampled pairs are labelled against the FP64 direct sum of each cluster.  Host outputs: feats
// (max_pairs x 8), labels (max_pairs), errs (max_pairs x 11, may be null: error / budget per order).
int tree_sample_labels(TreeSolver* t, const double4* src, const double4* tgt, int64_t stride, int64_t max_pairs,
                       float* feats, int32_t* labels, float* errs, int64_t* n_out) {
    if (!t->learned || max_pairs < 1 || max_pairs > (1 << 24) || !feats || !labels || !n_out) {
        set_error("tree_sample_labels: needs a LPM_ORDER_LEARNED solver, 1 <= max_pairs <= 2^24 and output arrays");
        return LPM_ERR_ARG;
    }
    *n_out = 0;
    if (t->n_src == 0 || t->n_tgt == 0) return LPM_OK;
    lpm_ctx* ctx = t->ctx;
    const int max_order = std::min(t->pm, kMlpDirectClass);
    TmpBuf bu, bp, bf, bl, be;
    LPM_CUDA_TRY(cudaMalloc(&bu.p, 3 * (size_t)t->n_tgt * sizeof(double)));
    LPM_CUDA_TRY(cudaMalloc(&bp.p, (size_t)max_pairs * sizeof(int2)));
    LPM_CUDA_TRY(cudaMalloc(&bf.p, (size_t)max_pairs * kMlpIn * sizeof(float)));
    LPM_CUDA_TRY(cudaMalloc(&bl.p, ((size_t)max_pairs + 1) * sizeof(int32_t)));
    LPM_CUDA_TRY(cudaMalloc(&be.p, (size_t)max_pairs * max_order * sizeof(float)));
    const bool had = t->mlp_loaded;
    const int32_t keep = t->ct.direct_below[t->order];
    t->mlp_loaded = false;
    t->ct.direct_below[t->order] = 1;
    int rc = tree_velocity(t, src, t->n_src, tgt, t->n_tgt, (double*)bu.p);
    t->ct.direct_below[t->order] = keep;
    t->mlp_loaded = had;
    if (rc) return rc;
    int32_t* dlab = (int32_t*)bl.p;
    int32_t* np_dev = dlab + max_pairs;  // count stored after the labels
    LPM_LAUNCH(ctx, "sample_pairs_kernel", sample_pairs_kernel, 64, 256, 0,
               t->far_off + (size_t)t->order * (t->n_batches + 1), t->tcount + 1, t->far_list,
               t->far_cap, t->flags + 2, stride, max_pairs, (int2*)bp.p, np_dev);
    const size_t smem = (size_t)entries_for(max_order) * sizeof(double4);
    if (smem > 48 * 1024)
        LPM_CUDA_TRY(cudaFuncSetAttribute(label_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    LPM_LAUNCH(ctx, "label_kernel", label_kernel, (unsigned)max_pairs, kBatch, smem, t->st, (const int2*)bp.p, np_dev,
               t->batch_first, t->tgt_sorted, t->src_sorted, t->batch_ctr, t->node_ctr, t->node_feat, t->node_wabs,
               t->B64, t->n_ent, t->gtab, t->ct, max_order, t->eps, (float*)bf.p, dlab, (float*)be.p);
    int32_t np = 0;
    LPM_CUDA_TRY(cudaMemcpyAsync(&np, np_dev, sizeof(int32_t), cudaMemcpyDeviceToHost, ctx->stream));
    LPM_CUDA_TRY(cudaStreamSynchronize(ctx->stream));
    LPM_CUDA_TRY(cudaMemcpyAsync(feats, bf.p, (size_t)np * kMlpIn * sizeof(float), cudaMemcpyDeviceToHost,
                                 ctx->stream));
    LPM_CUDA_TRY(cudaMemcpyAsync(labels, dlab, (size_t)np * sizeof(int32_t), cudaMemcpyDeviceToHost, ctx->stream));
    if (errs)
        LPM_CUDA_TRY(cudaMemcpyAsync(errs, be.p, (size_t)np * max_order * sizeof(float), cudaMemcpyDeviceToHost,
                                     ctx->stream));
    LPM_CUDA_TRY(cudaStreamSynchronize(ctx->stream));
    *n_out = np;
    return LPM_OK;
}

}  // namespace lpm
