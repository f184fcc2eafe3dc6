// Device octree with the reference's leaf membership.
//
// The reference builds its tree recursively (src/LpmTreeSum.cpp:266-290, src/LpmOctree.cpp:84-143):
// a node whose point count exceeds the leaf capacity is bisected at 0.5*(min+max) along all three
// axes in FP64 (src/LpmBox3d.cpp:140-151), points go to the child whose half-open box contains them
// (src/LpmBox3d.h:37-39), children are ordered ix + 2 iy + 4 iz and empty children are dropped.
//
// Here every point gets a 63-bit key that replays exactly those FP64 midpoint comparisons for 21
// levels (bit 63 set = outside the root box), the (key, index) pairs are radix sorted, and nodes are
// key ranges split level by level on the GPU: a node at level l with more than max_per_leaf points
// splits into the non-empty ranges of its points' level-(l+1) digits.  Sorted order is the
// reference's depth-first order, so leaves sorted by range start are its leaves in DFS order.
#include "octree.h"

#include <algorithm>

namespace lpm {

namespace {

constexpr int kSortThreads = 256;
constexpr int kSortItems = 16;
constexpr int kSortTile = kSortThreads * kSortItems;  // 4096 items per block
constexpr int kScanThreads = 256;
constexpr int kScanItems = 8;
constexpr int kScanTile = kScanThreads * kScanItems;

__device__ __forceinline__ int32_t warp_incl_scan(int32_t v) {
    const int lane = threadIdx.x & 31;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const int32_t t = __shfl_up_sync(0xffffffffu, v, o);
        if (lane >= o) v += t;
    }
    return v;
}

// Exclusive scan of one value per thread over a block of up to 1024 threads; returns the block total.
__device__ int32_t block_excl_scan(int32_t v, int32_t* total) {
    __shared__ int32_t warp_sums[32];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, nw = (blockDim.x + 31) >> 5;
    const int32_t incl = warp_incl_scan(v);
    if (lane == 31) warp_sums[w] = incl;
    __syncthreads();
    if (w == 0) {
        int32_t s = lane < nw ? warp_sums[lane] : 0;
        s = warp_incl_scan(s);
        if (lane < nw) warp_sums[lane] = s;
    }
    __syncthreads();
    const int32_t base = w ? warp_sums[w - 1] : 0;
    const int32_t tot = warp_sums[nw - 1];
    __syncthreads();
    if (total) *total = tot;
    return base + incl - v;
}

// ---------------------------------------------------------------------------------- scan
__global__ void scan_block_sums_kernel(const int32_t* __restrict__ in, int64_t n, int32_t* __restrict__ sums) {
    const int64_t base = (int64_t)blockIdx.x * kScanTile;
    int32_t s = 0;
#pragma unroll
    for (int k = 0; k < kScanItems; ++k) {
        const int64_t i = base + k * kScanThreads + threadIdx.x;
        if (i < n) s += in[i];
    }
    int32_t tot;
    block_excl_scan(s, &tot);
    if (threadIdx.x == 0) sums[blockIdx.x] = tot;
}

// In-place exclusive scan of m values by one block; writes the total to *total if given.
__global__ void scan_single_block_kernel(int32_t* __restrict__ data, int64_t m, int32_t* __restrict__ total) {
    const int64_t per = (m + blockDim.x - 1) / blockDim.x;
    const int64_t b = threadIdx.x * per, e = min(b + per, m);
    int32_t s = 0;
    for (int64_t i = b; i < e; ++i) s += data[i];
    int32_t tot;
    int32_t run = block_excl_scan(s, &tot);
    for (int64_t i = b; i < e; ++i) {
        const int32_t v = data[i];
        data[i] = run;
        run += v;
    }
    if (threadIdx.x == 0 && total) *total = tot;
}

__global__ void scan_apply_kernel(const int32_t* __restrict__ in, int32_t* __restrict__ out, int64_t n,
                                  const int32_t* __restrict__ sums) {
    const int64_t base = (int64_t)blockIdx.x * kScanTile + (int64_t)threadIdx.x * kScanItems;
    int32_t v[kScanItems];
    int32_t s = 0;
#pragma unroll
    for (int k = 0; k < kScanItems; ++k) {
        v[k] = base + k < n ? in[base + k] : 0;
        s += v[k];
    }
    int32_t run = block_excl_scan(s, nullptr) + sums[blockIdx.x];
#pragma unroll
    for (int k = 0; k < kScanItems; ++k) {
        if (base + k < n) out[base + k] = run;
        run += v[k];
    }
}

// ---------------------------------------------------------------------------------- radix sort
template <typename K>
__global__ void __launch_bounds__(kSortThreads) radix_hist_kernel(const K* __restrict__ keys, int64_t n, int shift,
                                                                  int32_t* __restrict__ counts, int nblocks) {
    __shared__ int32_t h[256];
    h[threadIdx.x] = 0;
    __syncthreads();
    const int64_t base = (int64_t)blockIdx.x * kSortTile;
#pragma unroll 4
    for (int k = 0; k < kSortItems; ++k) {
        const int64_t i = base + k * kSortThreads + threadIdx.x;
        if (i < n) atomicAdd(&h[(int)((keys[i] >> shift) & 255)], 1);
    }
    __syncthreads();
    counts[(int64_t)threadIdx.x * nblocks + blockIdx.x] = h[threadIdx.x];
}

// Stable scatter: warp w of a block owns items [w*512, (w+1)*512) of the block's tile and walks them
// in chunks of 32; __match_any_sync groups equal digits inside a chunk.
template <typename K>
__global__ void __launch_bounds__(kSortThreads) radix_scatter_kernel(const K* __restrict__ kin,
                                                                     const int32_t* __restrict__ vin,
                                                                     K* __restrict__ kout, int32_t* __restrict__ vout,
                                                                     int64_t n, int shift,
                                                                     const int32_t* __restrict__ offsets,
                                                                     int nblocks) {
    constexpr int kWarps = kSortThreads / 32;
    constexpr int kPerWarp = kSortTile / kWarps;
    __shared__ int32_t wh[kWarps][256];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    for (int d = threadIdx.x; d < kWarps * 256; d += kSortThreads) (&wh[0][0])[d] = 0;
    __syncthreads();
    const int64_t base = (int64_t)blockIdx.x * kSortTile + (int64_t)w * kPerWarp;
    const unsigned lt = (1u << lane) - 1u;
    for (int c = 0; c < kPerWarp / 32; ++c) {
        const int64_t i = base + c * 32 + lane;
        const bool valid = i < n;
        const int d = valid ? (int)((kin[i] >> shift) & 255) : 256;
        const unsigned peers = __match_any_sync(0xffffffffu, d);
        if (valid && lane == __ffs(peers) - 1) wh[w][d] += __popc(peers);
    }
    __syncthreads();
    {
        const int d = threadIdx.x;  // 256 threads, one per digit
        int32_t run = offsets[(int64_t)d * nblocks + blockIdx.x];
#pragma unroll
        for (int q = 0; q < kWarps; ++q) {
            const int32_t t = wh[q][d];
            wh[q][d] = run;
            run += t;
        }
    }
    __syncthreads();
    for (int c = 0; c < kPerWarp / 32; ++c) {
        const int64_t i = base + c * 32 + lane;
        const bool valid = i < n;
        K key = 0;
        int d = 256;
        if (valid) {
            key = kin[i];
            d = (int)((key >> shift) & 255);
        }
        const unsigned peers = __match_any_sync(0xffffffffu, d);
        const int32_t pos = valid ? wh[w][d] + __popc(peers & lt) : 0;
        __syncwarp();
        if (valid) {
            kout[pos] = key;
            vout[pos] = vin[i];
            if (lane == __ffs(peers) - 1) wh[w][d] += __popc(peers);
        }
        __syncwarp();
    }
}

template <typename K>
int radix_sort_impl(lpm_ctx* ctx, K* keys, int32_t* vals, K* tk, int32_t* tv, int64_t n, int bit_lo, int bit_hi,
                    int counts_slot, int sums_slot) {
    if (n <= 1) return LPM_OK;
    const int nblocks = (int)((n + kSortTile - 1) / kSortTile);
    int32_t* counts = (int32_t*)scratch(ctx, counts_slot, sizeof(int32_t) * 256 * (size_t)nblocks);
    if (!counts) return LPM_ERR_OOM;
    K* src_k = keys;
    int32_t* src_v = vals;
    K* dst_k = tk;
    int32_t* dst_v = tv;
    for (int shift = bit_lo; shift < bit_hi; shift += 8) {
        LPM_LAUNCH(ctx, "radix_hist_kernel", radix_hist_kernel<K>, nblocks, kSortThreads, 0, src_k, n, shift, counts,
                   nblocks);
        // digit-major counts -> global offsets; a single block suffices for small arrays, the three-pass
        // scan takes the large ones (1.3M keys: 256 x 1280 counts)
        if ((int64_t)256 * nblocks <= 16 * 1024) {
            LPM_LAUNCH(ctx, "scan_single_block_kernel", scan_single_block_kernel, 1, 1024, 0, counts,
                       (int64_t)256 * nblocks, (int32_t*)nullptr);
        } else {
            const int rc = scan_exclusive_i32(ctx, counts, counts, (int64_t)256 * nblocks, nullptr, sums_slot);
            if (rc) return rc;
        }
        LPM_LAUNCH(ctx, "radix_scatter_kernel", radix_scatter_kernel<K>, nblocks, kSortThreads, 0, src_k, src_v, dst_k,
                   dst_v, n, shift, counts, nblocks);
        std::swap(src_k, dst_k);
        std::swap(src_v, dst_v);
    }
    if (src_k != keys) {
        LPM_CUDA_TRY(cudaMemcpyAsync(keys, src_k, sizeof(K) * (size_t)n, cudaMemcpyDeviceToDevice, ctx->stream));
        LPM_CUDA_TRY(cudaMemcpyAsync(vals, src_v, sizeof(int32_t) * (size_t)n, cudaMemcpyDeviceToDevice, ctx->stream));
    }
    return LPM_OK;
}

// ---------------------------------------------------------------------------------- keys
__global__ void morton_keys_kernel(const double4* __restrict__ pts, int64_t n, RootBox root,
                                   uint64_t* __restrict__ keys, int32_t* __restrict__ vals,
                                   int32_t* __restrict__ counters, int bits, int max_depth) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    root = resolve_root(root);
    bool in = false;
    if (i < n) {
        const double4 p = pts[i];
        const double c[3] = {p.x, p.y, p.z};
        in = root.lo[0] <= c[0] && c[0] < root.hi[0] && root.lo[1] <= c[1] && c[1] < root.hi[1] &&
             root.lo[2] <= c[2] && c[2] < root.hi[2];
        uint64_t key = kKeyOutside;
        if (in && bits == 1) {  // binary: level l bisects axis (l + 1) mod 3 (the Sakajo tree's (j + 2) mod 3, j = l - 1)
            double lo[3] = {root.lo[0], root.lo[1], root.lo[2]};
            double hi[3] = {root.hi[0], root.hi[1], root.hi[2]};
            key = 0;
            for (int l = 1; l <= max_depth; ++l) {
                const int a = (l + 1) % 3;
                const double mid = 0.5 * (lo[a] + hi[a]);  // Box3d::bisectAlongDims midpoint
                if (c[a] < mid) {
                    hi[a] = mid;
                } else {
                    lo[a] = mid;
                    key |= 1ull << (kMaxLevels - l);
                }
            }
        } else if (in) {
            double lo[3] = {root.lo[0], root.lo[1], root.lo[2]};
            double hi[3] = {root.hi[0], root.hi[1], root.hi[2]};
            key = 0;
            for (int l = 1; l <= kKeyLevels; ++l) {
                uint64_t digit = 0;
#pragma unroll
                for (int a = 0; a < 3; ++a) {
                    const double mid = 0.5 * (lo[a] + hi[a]);  // Box3d::bisectAll midpoint
                    if (c[a] < mid) {
                        hi[a] = mid;
                    } else {
                        lo[a] = mid;
                        digit |= 1ull << a;
                    }
                }
                key |= digit << (3 * (kKeyLevels - l));
            }
        }
        keys[i] = key;
        vals[i] = (int32_t)i;
    }
    const unsigned b = __ballot_sync(0xffffffffu, in);
    if ((threadIdx.x & 31) == 0 && b) atomicAdd(&counters[0], __popc(b));
}

__global__ void root_extent_kernel(const double4* __restrict__ pts, int64_t first, int64_t n, int mode,
                                   unsigned long long* __restrict__ r_dev) {
    unsigned long long m = 0;  // non-negative doubles order like their bit patterns
    for (int64_t i = first + (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
         i += (int64_t)gridDim.x * blockDim.x) {
        const double4 p = pts[i];
        const double v = mode == kRootMaxNorm ? fmax(fabs(p.x), fmax(fabs(p.y), fabs(p.z)))
                                              : __dadd_rn(__dadd_rn(__dmul_rn(p.x, p.x), __dmul_rn(p.y, p.y)),
                                                          __dmul_rn(p.z, p.z));
        const unsigned long long b = (unsigned long long)__double_as_longlong(v);
        m = b > m ? b : m;
    }
    for (int o = 16; o > 0; o >>= 1) {
        const unsigned long long u = __shfl_xor_sync(0xffffffffu, m, o);
        m = u > m ? u : m;
    }
    if ((threadIdx.x & 31) == 0 && m) atomicMax(r_dev, m);
}

__device__ __forceinline__ int level_digit(uint64_t key, int level, int bits) {
    return bits == 1 ? (int)((key >> (kMaxLevels - level)) & 1ull) : (int)((key >> (3 * (kKeyLevels - level))) & 7ull);
}

// Box of child digit d of a level-l node (box pb): all three axes for octrees (ix + 2 iy + 4 iz), axis
// (l + 2) mod 3 for binary trees.
__device__ __forceinline__ void child_box(const double* pb, int l, int d, int bits, double* cb) {
    for (int a = 0; a < 3; ++a) {
        const double mid = 0.5 * (pb[2 * a] + pb[2 * a + 1]);
        const bool split = bits == 3 || a == (l + 2) % 3;
        const bool upper = bits == 3 ? ((d >> a) & 1) : (d & 1);
        cb[2 * a] = split && upper ? mid : pb[2 * a];
        cb[2 * a + 1] = split && !upper ? mid : pb[2 * a + 1];
    }
}

// Box3d::intersectsSphere about the origin (src/LpmBox3d.cpp:79-129): the box's closest point lies inside
// the sphere and its farthest corner outside (distances sqrt((x x + y y) + z z), rounded step by step).
__device__ __forceinline__ double mag3(double x, double y, double z) {
    return __dsqrt_rn(__dadd_rn(__dadd_rn(__dmul_rn(x, x), __dmul_rn(y, y)), __dmul_rn(z, z)));
}
__device__ bool box_meets_sphere(const double* b, double r) {
    double c[3];
    const bool inside = b[0] <= 0.0 && 0.0 < b[1] && b[2] <= 0.0 && 0.0 < b[3] && b[4] <= 0.0 && 0.0 < b[5];
    for (int a = 0; a < 3; ++a) {
        const double lo = b[2 * a], hi = b[2 * a + 1];
        c[a] = inside ? 0.0 : (lo == hi ? lo : (lo >= 0.0 ? lo : (hi <= 0.0 ? hi : 0.0)));
    }
    double far = 0.0;
    for (int k = 0; k < 8; ++k) {
        const double d = mag3(b[(k & 1) ? 1 : 0], b[(k & 2) ? 3 : 2], b[(k & 4) ? 5 : 4]);
        far = d > far ? d : far;
    }
    return mag3(c[0], c[1], c[2]) <= r && far >= r;
}

__global__ void tree_init_kernel(Octree t) {
    t.node_start[0] = 0;
    t.node_end[0] = t.counters[0];
    t.node_parent[0] = -1;
    t.node_first_child[0] = -1;
    t.node_nchild[0] = 0;
    t.node_level[0] = 0;
    const RootBox root = resolve_root(t.root);
    for (int a = 0; a < 3; ++a) {
        t.node_box[2 * a] = root.lo[a];
        t.node_box[2 * a + 1] = root.hi[a];
    }
    t.level_range[0] = 0;
    t.level_range[1] = 1;
    for (int l = 1; l < kMaxLevels + 2; ++l) {
        t.level_range[2 * l] = 1;
        t.level_range[2 * l + 1] = 1;
    }
    t.counters[1] = 1;
    t.counters[2] = 0;
    t.counters[4] = 0;
}

// For each node of level l holding more than max_per_leaf points: the 9 boundaries of its
// level-(l+1) digit ranges, and the number of non-empty children.
__global__ void __launch_bounds__(256) split_level_kernel(Octree t, int l) {
    // One block per node (grid-stride over the level): warp d (1..7) finds the first position of the node's
    // sorted key range whose level-(l+1) digit is >= d by a 32-ary search (32 probes per round, ~4 rounds
    // for a million keys instead of ~20 dependent probes of a binary search).
    __shared__ int cs_sh[9];
    const int lb = t.level_range[2 * l], le = t.level_range[2 * l + 1];
    const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const unsigned full = 0xffffffffu;
    const int nd = 1 << t.bits;  // digits per level
    for (int i = lb + blockIdx.x; i < le; i += gridDim.x) {
        const int s = t.node_start[i], e = t.node_end[i];
        const bool split = e - s > t.max_per_leaf;  // uniform per block
        if (split) {
            if (w >= 1 && w < nd) {
                const int d = w;
                int lo = s, hi = e;  // the boundary b satisfies lo <= b <= hi; positions lo..hi-1 are keys
                while (hi - lo > 32) {
                    const int64_t L = hi - lo;
                    const int p = lo + (int)(((int64_t)lane * L) >> 5);
                    const unsigned below = __ballot_sync(full, level_digit(t.keys[p], l + 1, t.bits) < d);
                    const int c = __popc(below);  // probes 0..c-1 lie below the boundary (digits are sorted)
                    const int nlo = c == 0 ? lo : lo + (int)(((int64_t)(c - 1) * L) >> 5) + 1;
                    const int nhi = c == 32 ? hi : lo + (int)(((int64_t)c * L) >> 5);
                    lo = nlo;
                    hi = nhi;
                }
                const bool lt = lane < hi - lo && level_digit(t.keys[lo + lane], l + 1, t.bits) < d;
                const int c = __popc(__ballot_sync(full, lt));
                if (lane == 0) cs_sh[d] = lo + c;
            } else if (w == 0 && lane == 0) {
                cs_sh[0] = s;
                cs_sh[nd] = e;
            }
        }
        __syncthreads();
        if (threadIdx.x == 0) {
            int nchild = 0;
            if (split) {
                int32_t* cs = t.child_start + (int64_t)(i - lb) * 9;
                for (int d = 0; d <= nd; ++d) cs[d] = cs_sh[d];
                for (int d = 0; d < nd; ++d) {
                    bool keep = cs_sh[d + 1] > cs_sh[d];
                    if (keep && t.sphere_r > 0.0) {
                        double cb[6];
                        child_box(t.node_box + 6 * (int64_t)i, l, d, t.bits, cb);
                        keep = box_meets_sphere(cb, t.sphere_r);
                    }
                    nchild += keep;
                }
            }
            t.node_split[i - lb] = nchild;
        }
        __syncthreads();  // cs_sh is reused by the next node
    }
}

// One block: scan the level's child counts and append the children as level l+1.
__global__ void emit_level_kernel(Octree t, int l) {
    __shared__ int32_t s_total;
    const int lb = t.level_range[2 * l], le = t.level_range[2 * l + 1];
    const int m = le - lb;
    const int per = (m + blockDim.x - 1) / blockDim.x;
    const int b = threadIdx.x * per, e = min(b + per, m);
    int32_t s = 0;
    for (int i = b; i < e; ++i) s += t.node_split[i];
    int32_t tot;
    int32_t run = block_excl_scan(s, &tot) + le;
    if (threadIdx.x == 0) s_total = tot;
    for (int i = b; i < e; ++i) {
        const int node = lb + i;
        const int nc = t.node_split[i];
        if (nc == 0 || run + nc > t.node_cap) {
            if (nc > 0) atomicOr(&t.counters[2], 2);  // node capacity exhausted
            t.node_first_child[node] = -1;
            t.node_nchild[node] = 0;
            continue;
        }
        t.node_first_child[node] = run;
        t.node_nchild[node] = (int8_t)nc;
        const int32_t* cs = t.child_start + (int64_t)i * 9;
        const double* pb = t.node_box + 6 * (int64_t)node;
        int k = run;
        for (int d = 0; d < (1 << t.bits); ++d) {
            if (cs[d + 1] <= cs[d]) continue;
            double cb[6];
            child_box(pb, l, d, t.bits, cb);
            if (t.sphere_r > 0.0 && !box_meets_sphere(cb, t.sphere_r)) continue;  // as counted by split_level
            t.node_start[k] = cs[d];
            t.node_end[k] = cs[d + 1];
            t.node_parent[k] = node;
            t.node_first_child[k] = -1;
            t.node_nchild[k] = 0;
            t.node_level[k] = (int8_t)(l + 1);
            for (int a = 0; a < 6; ++a) t.node_box[6 * (int64_t)k + a] = cb[a];
            ++k;
        }
        run += nc;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        const int tot2 = (int)min((int64_t)s_total, t.node_cap - (int64_t)le);
        t.level_range[2 * (l + 1)] = le;
        t.level_range[2 * (l + 1) + 1] = le + max(tot2, 0);
        t.counters[1] = le + max(tot2, 0);
        if (tot2 > 0) t.counters[4] = l + 1;
    }
}

__global__ void leaf_flags_kernel(Octree t, int64_t n) {
    const int nn = t.counters[1];
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < nn; i += gridDim.x * blockDim.x) {
        if (t.node_nchild[i] == 0) {
            t.leaf_flag[t.node_start[i]] = 1;
            if (t.max_per_leaf > 0 && t.node_end[i] - t.node_start[i] > t.max_per_leaf)
                atomicOr(&t.counters[2], 1);  // depth limit
        }
    }
    (void)n;
}

__global__ void leaf_ids_kernel(Octree t, int64_t n) {
    const int nn = t.counters[1];
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < nn; i += gridDim.x * blockDim.x) {
        if (t.node_nchild[i] == 0) {
            const int leaf = t.leaf_flag[t.node_start[i]];
            t.node_leaf[i] = leaf;
            t.leaf_node[leaf] = i;
        } else {
            t.node_leaf[i] = -1;
        }
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) t.counters[3] = t.leaf_flag[n];
}

__global__ void fill_i32_kernel(int32_t* p, int64_t n, int32_t v) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) p[i] = v;
}

}  // namespace

int scan_exclusive_i32(lpm_ctx* ctx, const int32_t* in, int32_t* out, int64_t n, int32_t* total_dev, int sums_slot) {
    if (n <= 0) return LPM_OK;
    const int nblocks = (int)((n + kScanTile - 1) / kScanTile);
    int32_t* sums = (int32_t*)scratch(ctx, sums_slot, sizeof(int32_t) * (size_t)(nblocks + 1));
    if (!sums) return LPM_ERR_OOM;
    LPM_LAUNCH(ctx, "scan_block_sums_kernel", scan_block_sums_kernel, nblocks, kScanThreads, 0, in, n, sums);
    LPM_LAUNCH(ctx, "scan_single_block_kernel", scan_single_block_kernel, 1, 1024, 0, sums, (int64_t)nblocks,
               total_dev);
    LPM_LAUNCH(ctx, "scan_apply_kernel", scan_apply_kernel, nblocks, kScanThreads, 0, in, out, n, sums);
    return LPM_OK;
}

int morton_keys(lpm_ctx* ctx, const double4* pts, int64_t n, const RootBox& root, uint64_t* keys, int32_t* vals,
                int32_t* counter) {
    if (n <= 0) return LPM_OK;
    LPM_LAUNCH(ctx, "morton_keys_kernel", morton_keys_kernel, grid_for(n, 256), 256, 0, pts, n, root, keys, vals,
               counter, 3, kKeyLevels);
    return LPM_OK;
}

int root_extent(lpm_ctx* ctx, const double4* pts, int64_t first, int64_t n, int mode, unsigned long long* r_dev) {
    LPM_CUDA_TRY(cudaMemsetAsync(r_dev, 0, sizeof(unsigned long long), ctx->stream));
    if (n <= first) return LPM_OK;
    const unsigned g = (unsigned)std::max<int64_t>(1, std::min<int64_t>(grid_for(n - first, 256), 2 * ctx->num_sms));
    LPM_LAUNCH(ctx, "root_extent_kernel", root_extent_kernel, g, 256, 0, pts, first, n, mode, r_dev);
    return LPM_OK;
}

int radix_sort_u64(lpm_ctx* ctx, uint64_t* keys, int32_t* vals, uint64_t* tk, int32_t* tv, int64_t n, int bit_lo,
                   int counts_slot, int sums_slot) {
    return radix_sort_impl<uint64_t>(ctx, keys, vals, tk, tv, n, bit_lo, 64, counts_slot, sums_slot);
}

int radix_sort_u32(lpm_ctx* ctx, uint32_t* keys, int32_t* vals, uint32_t* tk, int32_t* tv, int64_t n, int bits) {
    return radix_sort_impl<uint32_t>(ctx, keys, vals, tk, tv, n, 0, bits, kSlotMisc1, kSlotMisc2);
}

int octree_alloc(Octree& t, int64_t n, int max_per_leaf, int max_depth, int bits, double sphere_r) {
    octree_free(t);
    t.n = n;
    t.max_per_leaf = max_per_leaf;
    t.bits = bits == 1 ? 1 : 3;
    t.levels = t.bits == 1 ? kMaxLevels : kKeyLevels;
    t.max_depth = std::min(std::max(max_depth, 1), t.levels);
    t.sphere_r = t.bits == 1 ? sphere_r : 0.0;
    if (t.bits == 1) {
        // every non-empty node splits to max_depth: level l holds at most min(n, 2^l) nodes
        int64_t cap = 0;
        for (int l = 0; l <= t.max_depth; ++l) cap += l < 62 ? std::min<int64_t>(n, 1ll << l) : n;
        t.node_cap = cap + 16;
    } else {
        // every internal node has >= 2 points in distinct children or splits a range of > max points:
        // n_nodes <= 8 * (internal nodes) + 1 and internal nodes <= depth * n / (max_per_leaf + 1) + 1
        const int64_t internal = (int64_t)t.max_depth * (n / (max_per_leaf + 1) + 1) + 1;
        t.node_cap = std::min<int64_t>(8 * internal + 1, std::max<int64_t>(2 * n + 16, 64));
    }
    const size_t nn = (size_t)std::max<int64_t>(n, 1), nc = (size_t)t.node_cap;
    cudaError_t e = cudaSuccess;
    auto A = [&](void** p, size_t bytes) {
        if (e == cudaSuccess) e = dev_alloc((void**)p, bytes);
    };
    A((void**)&t.keys, nn * 8);
    A((void**)&t.perm, nn * 4);
    A((void**)&t.tmp_keys, nn * 8);
    A((void**)&t.tmp_vals, nn * 4);
    A((void**)&t.leaf_flag, (nn + 1) * 4);
    A((void**)&t.node_start, nc * 4);
    A((void**)&t.node_end, nc * 4);
    A((void**)&t.node_parent, nc * 4);
    A((void**)&t.node_first_child, nc * 4);
    A((void**)&t.node_nchild, nc);
    A((void**)&t.node_level, nc);
    A((void**)&t.node_box, nc * 6 * 8);
    A((void**)&t.node_split, nc * 4);
    A((void**)&t.child_start, nc * 9 * 4);
    A((void**)&t.level_range, 2 * (kMaxLevels + 2) * 4);
    A((void**)&t.counters, 16 * 4);
    A((void**)&t.leaf_node, nc * 4);
    A((void**)&t.node_leaf, nc * 4);
    if (e != cudaSuccess) {
        octree_free(t);
        return cuda_status(e, "cudaMalloc (octree)");
    }
    return LPM_OK;
}

void octree_free(Octree& t) {
    void* ps[] = {t.keys, t.perm, t.tmp_keys, t.tmp_vals, t.leaf_flag, t.node_start, t.node_end, t.node_parent,
                  t.node_first_child, t.node_nchild, t.node_level, t.node_box, t.node_split, t.child_start,
                  t.level_range, t.counters, t.leaf_node, t.node_leaf};
    for (void* p : ps)
        if (p) cudaFree(p);
    const Octree keep = t;
    t = Octree();
    t.n = keep.n;
    t.max_per_leaf = keep.max_per_leaf;
    t.max_depth = keep.max_depth;
    t.bits = keep.bits;
    t.levels = keep.levels;
    t.sphere_r = keep.sphere_r;
}

int octree_build(lpm_ctx* ctx, Octree& t, const double4* pts, int64_t n, const RootBox& root) {
    if (n > t.n || n >= INT32_MAX) {
        set_error("octree_build: %lld points exceed the tree's capacity", (long long)n);
        return LPM_ERR_CAPACITY;
    }
    t.root = root;
    LPM_CUDA_TRY(cudaMemsetAsync(t.counters, 0, 16 * 4, ctx->stream));
    if (n > 0)
        LPM_LAUNCH(ctx, "morton_keys_kernel", morton_keys_kernel, grid_for(n, 256), 256, 0, pts, n, root, t.keys,
                   t.perm, t.counters, t.bits, t.max_depth);
    // the key bits that decide levels 1..max_depth (and the outside flag in bit 63)
    const int bit_lo = std::max(0, t.bits * (t.levels - t.max_depth)) & ~7;
    int rc = radix_sort_u64(ctx, t.keys, t.perm, t.tmp_keys, t.tmp_vals, n, bit_lo);
    if (rc) return rc;
    LPM_LAUNCH(ctx, "tree_init_kernel", tree_init_kernel, 1, 1, 0, t);
    const unsigned sgrid = (unsigned)std::max<int64_t>(1, std::min<int64_t>(grid_for(t.node_cap, 256),
                                                                             4 * ctx->num_sms));
    const unsigned split_grid = (unsigned)std::max<int64_t>(1, std::min<int64_t>(t.node_cap, 8 * ctx->num_sms));
    for (int l = 0; l < t.max_depth; ++l) {
        LPM_LAUNCH(ctx, "split_level_kernel", split_level_kernel, split_grid, 256, 0, t, l);
        LPM_LAUNCH(ctx, "emit_level_kernel", emit_level_kernel, 1, 1024, 0, t, l);
    }
    LPM_LAUNCH(ctx, "fill_i32_kernel", fill_i32_kernel, grid_for(n + 1, 256), 256, 0, t.leaf_flag, n + 1, 0);
    LPM_LAUNCH(ctx, "leaf_flags_kernel", leaf_flags_kernel, sgrid, 256, 0, t, n);
    rc = scan_exclusive_i32(ctx, t.leaf_flag, t.leaf_flag, n + 1, nullptr);
    if (rc) return rc;
    LPM_LAUNCH(ctx, "leaf_ids_kernel", leaf_ids_kernel, sgrid, 256, 0, t, n);
    return LPM_OK;
}

}  // namespace lpm
