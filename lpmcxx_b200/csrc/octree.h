// Device octree: Morton keys that replay the reference's FP64 midpoint bisection, an LSD radix
// sort, and a level-synchronous split of key ranges into nodes.
#pragma once

#include "lpm_internal.h"

namespace lpm {

constexpr int kKeyLevels = 21;        // 3 bits per level in a 63-bit key; bit 63 marks "outside the root box"
constexpr int kMaxLevels = 63;        // binary (1 bit per level) trees: up to 63 levels
constexpr uint64_t kKeyOutside = ~0ull;

// Exclusive prefix sum of n int32 values (in may equal out).  Uses ctx scratch slot `sums_slot`.
int scan_exclusive_i32(lpm_ctx* ctx, const int32_t* in, int32_t* out, int64_t n, int32_t* total_dev,
                       int sums_slot = kSlotMisc2);

// Stable LSD radix sort of (key, value) pairs over key bits [bit_lo, 64), 8 bits per pass.
// keys/vals are sorted in place (ping-pong through tmp_keys/tmp_vals, which must hold n items).  Digit counts
// go to ctx scratch slot `counts_slot`, scan sums to `sums_slot` (sorts on concurrent streams use distinct slots).
int radix_sort_u64(lpm_ctx* ctx, uint64_t* keys, int32_t* vals, uint64_t* tmp_keys, int32_t* tmp_vals, int64_t n,
                   int bit_lo, int counts_slot = kSlotMisc1, int sums_slot = kSlotMisc2);
int radix_sort_u32(lpm_ctx* ctx, uint32_t* keys, int32_t* vals, uint32_t* tmp_keys, int32_t* tmp_vals, int64_t n,
                   int bits);

// Root box of a build.  With r_dev set, the box is computed on the device when the build runs (so a
// captured graph follows the points): r_dev holds the bit pattern of a non-negative double r (written by
// root_extent) and the box is Box3d(R) with its padding, [-R - 1e-5, R + 1e-5]^3 (src/LpmBox3d.h:21-33),
// R = sqrt(r) for kRootEuclid (Coords::maxR, src/LpmCoords.cpp:136-143) or R = r for kRootMaxNorm.
constexpr int kRootEuclid = 0;
constexpr int kRootMaxNorm = 1;
struct RootBox {
    double lo[3], hi[3];
    const unsigned long long* r_dev = nullptr;
    int mode = kRootEuclid;
};

#ifdef __CUDACC__
__device__ __forceinline__ RootBox resolve_root(const RootBox& r) {
    if (!r.r_dev) return r;
    RootBox b = r;
    const double v = __longlong_as_double((long long)*r.r_dev);
    const double R = r.mode == kRootMaxNorm ? v : sqrt(v);
    for (int a = 0; a < 3; ++a) {
        b.lo[a] = -R - 1e-5;
        b.hi[a] = R + 1e-5;
    }
    b.r_dev = nullptr;
    return b;
}
#endif

// *r_dev = max over pts[first:n] of (x x + y y) + z z (rounded as Coords::maxR: no fused multiply-add) for
// kRootEuclid, or of max(|x|, |y|, |z|) for kRootMaxNorm, as the bit pattern of the double.  Capturable.
int root_extent(lpm_ctx* ctx, const double4* pts, int64_t first, int64_t n, int mode, unsigned long long* r_dev);

// Octree over points (double4, xyz used).  All arrays device-resident; sizes are capacities.
// bits = 3: every level bisects all three axes (8 children, child order ix + 2 iy + 4 iz); nodes holding more
// than max_per_leaf points split.  bits = 1: the Sakajo (2009) tree (src/LpmSakajo2009.cpp:25-63): level l
// bisects axis (l + 2) mod 3 (z, x, y, z, ...), every non-empty node splits down to max_depth
// (max_per_leaf = 0), and with sphere_r > 0 a child is kept only if its box meets the sphere of that radius
// about the origin (Box3d::intersectsSphere, src/LpmBox3d.cpp:125-129).
struct Octree {
    int64_t n = 0;          // points given
    int max_per_leaf = 0;
    int max_depth = 0;      // levels the keys are split to (<= levels)
    int bits = 3;           // key bits per level: 3 (octree) or 1 (binary, axis-cycling)
    int levels = kKeyLevels;  // levels a key holds: 63 / bits
    double sphere_r = 0.0;  // binary trees: keep children that meet this sphere (0: keep every non-empty one)
    int64_t node_cap = 0;
    RootBox root{};
    // per point (sorted order)
    uint64_t* keys = nullptr;      // sorted keys
    int32_t* perm = nullptr;       // sorted position -> original index
    uint64_t* tmp_keys = nullptr;
    int32_t* tmp_vals = nullptr;
    // per node (level order)
    int32_t* node_start = nullptr;
    int32_t* node_end = nullptr;
    int32_t* node_parent = nullptr;
    int32_t* node_first_child = nullptr;  // -1 for a leaf
    int8_t* node_nchild = nullptr;
    int8_t* node_level = nullptr;
    double* node_box = nullptr;           // 6 per node: xlo, xhi, ylo, yhi, zlo, zhi
    int32_t* node_split = nullptr;        // scratch: child counts of a level
    int32_t* child_start = nullptr;       // scratch: 9 boundaries per node of a level
    int32_t* level_range = nullptr;       // [2 * (kKeyLevels + 2)]: begin/end of each level's nodes
    int32_t* counters = nullptr;          // [0] n_valid, [1] n_nodes, [2] overflow flag, [3] n_leaves, [4] depth
    // leaves in depth-first order
    int32_t* leaf_node = nullptr;         // leaf index -> node id
    int32_t* node_leaf = nullptr;         // node id -> leaf index (or -1)
    int32_t* leaf_flag = nullptr;         // scratch over points
};

// keys[i], vals[i] = i for pts[0:n]; counter[0] += number of points inside the root box.
int morton_keys(lpm_ctx* ctx, const double4* pts, int64_t n, const RootBox& root, uint64_t* keys, int32_t* vals,
                int32_t* counter);

int octree_alloc(Octree& t, int64_t n, int max_per_leaf, int max_depth, int bits = 3, double sphere_r = 0.0);
void octree_free(Octree& t);
// Build over pts[0:n] with the given root box.  Fully asynchronous (capturable): no host reads.
int octree_build(lpm_ctx* ctx, Octree& t, const double4* pts, int64_t n, const RootBox& root);

}  // namespace lpm
