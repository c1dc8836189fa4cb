// Sort-based contact detection for one large scene (whole GPU): sweep and prune
// along x over bodies sorted by AABB min-x, candidate pairs sorted by
// (id0, id1) so the contact order is the reference's (DynamicSystem.cpp:262-276),
// then a counting pass, an exclusive scan and a writing pass of the same
// narrow phase and merge as the per-scene kernel.  Replaces FCL's dynamic AABB
// tree broad phase (src/Contact/BroadPhase.cpp:6-10) for scenes with thousands
// of bodies.
#pragma once
#include <cub/device/device_radix_sort.cuh>
#include <cub/device/device_scan.cuh>

#include "pdc_collide.cuh"

namespace pdc {

struct LargeCollide {
    int nb_max;           // bodies of the largest large scene
    long long max_pairs;  // candidate pair capacity
    unsigned int* key;    // [nb_max] orderable min-x
    int* val;             // [nb_max] body (scene-local)
    unsigned int* key_s;
    int* val_s;
    float* box;           // [nb_max][6] AABB (minx, maxx, miny, maxy, minz, maxz), body order
    unsigned long long* pairs;    // [max_pairs] (lo << 32) | hi, unused = ~0
    unsigned long long* pairs_s;
    int* npairs;          // [1] candidate pairs emitted
    int* overflow;        // [1] candidate pairs dropped
    int* cnt;             // [max_pairs] contact points per pair
    int* off;             // [max_pairs] exclusive prefix
    void* temp;           // CUB temporary storage
    size_t temp_bytes;
};

__device__ __forceinline__ unsigned int orderable(float f) {
    const unsigned int u = __float_as_uint(f);
    return (u & 0x80000000u) ? ~u : (u | 0x80000000u);
}

// AABBs (slightly widened so float rounding never hides an overlap) and sort keys
__global__ void large_aabb_kernel(const __grid_constant__ WorldPtrs W, LargeCollide L, int scene) {
    const int b0 = W.body_off[scene], nb = W.body_off[scene + 1] - b0;
    for (int b = blockIdx.x * blockDim.x + threadIdx.x; b < nb; b += gridDim.x * blockDim.x) {
        const BodyG g = load_body(W, b0 + b);
        float lo[3], hi[3];
        if (g.type == SHAPE_PLANE) {
            for (int r = 0; r < 3; ++r) {
                lo[r] = -INFINITY;
                hi[r] = INFINITY;
            }
        } else {
            const double c[3] = {g.c.x, g.c.y, g.c.z};
            for (int r = 0; r < 3; ++r) {
                const double e = (g.type == SHAPE_SPHERE)
                                     ? g.h[0]
                                     : fabs(g.R[3 * r]) * g.h[0] + fabs(g.R[3 * r + 1]) * g.h[1] +
                                           fabs(g.R[3 * r + 2]) * g.h[2];
                const double pad = 1e-6 * (e + fabs(c[r]));
                lo[r] = __double2float_rd(c[r] - e - pad);
                hi[r] = __double2float_ru(c[r] + e + pad);
            }
        }
        float* bx = L.box + 6 * b;
        bx[0] = lo[0]; bx[1] = hi[0]; bx[2] = lo[1]; bx[3] = hi[1]; bx[4] = lo[2]; bx[5] = hi[2];
        L.key[b] = orderable(lo[0]);
        L.val[b] = b;
    }
}

// sweep: body at sorted position i against the following bodies whose min-x
// does not exceed its max-x; overlapping (not both static) pairs are emitted
__global__ void large_sweep_kernel(const __grid_constant__ WorldPtrs W, LargeCollide L, int scene) {
    const int b0 = W.body_off[scene], nb = W.body_off[scene + 1] - b0;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < nb; i += gridDim.x * blockDim.x) {
        const int a = L.val_s[i];
        const float* ba = L.box + 6 * a;
        const unsigned int kmax = orderable(ba[1]);
        const bool sa = W.is_static[b0 + a] != 0;
        for (int j = i + 1; j < nb && L.key_s[j] <= kmax; ++j) {
            const int c = L.val_s[j];
            if (sa && W.is_static[b0 + c]) continue;
            const float* bc = L.box + 6 * c;
            if (bc[2] > ba[3] || ba[2] > bc[3] || bc[4] > ba[5] || ba[4] > bc[5]) continue;
            const unsigned int lo = min(a, c), hi = max(a, c);
            const int slot = atomicAdd(L.npairs, 1);
            if (slot < L.max_pairs) L.pairs[slot] = ((unsigned long long)lo << 32) | hi;
            else atomicAdd(L.overflow, 1);
        }
    }
}

// narrow phase of the sorted candidate pairs; pass 0 counts, pass 1 writes
__global__ void large_narrow_kernel(const __grid_constant__ WorldPtrs W, LargeCollide L, int scene, int pass) {
    const int b0 = W.body_off[scene];
    const int cap0 = W.contact_cap[scene], cap = W.contact_cap[scene + 1] - cap0;
    const long long np = min((long long)*L.npairs, L.max_pairs);
    for (long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x; p < L.max_pairs;
         p += (long long)gridDim.x * blockDim.x) {
        if (p >= np) {
            if (!pass) L.cnt[p] = 0;
            continue;
        }
        const unsigned long long key = L.pairs_s[p];
        const int i = (int)(key >> 32), j = (int)(key & 0xffffffffu);
        const BodyG A = load_body(W, b0 + i), Bg = load_body(W, b0 + j);
        CPoint pts[PDC_MAX_PAIR_POINTS];
        int m = pair_points(A, Bg, pts);
        m = merge_points(pts, m);
        if (!pass) {
            L.cnt[p] = m;
            continue;
        }
        int off = L.off[p];
        for (int q = 0; q < m; ++q, ++off) {
            if (off >= cap) continue;
            const long long gc = cap0 + off;
            W.cbody[2 * gc] = i;
            W.cbody[2 * gc + 1] = j;
            frame_from_normal(pts[q].n, W.frame + 9 * gc);
            st3(W.arm + 6 * gc, sub3(pts[q].p, A.c));
            st3(W.arm + 6 * gc + 3, sub3(pts[q].p, Bg.c));
            W.depth[gc] = fabs(pts[q].depth);
            st3(W.cpos + 3 * gc, pts[q].p);
        }
    }
}

__global__ void large_total_kernel(const __grid_constant__ WorldPtrs W, LargeCollide L, int scene) {
    const int cap = W.contact_cap[scene + 1] - W.contact_cap[scene];
    const long long last = L.max_pairs - 1;
    const long long total = (long long)L.off[last] + L.cnt[last];
    if (W.dt[scene] == 0.0) {  // done with its adaptive substeps
        W.ccount[scene] = 0;
        W.overflow[scene] = 0;
        return;
    }
    W.ccount[scene] = (int)min(total, (long long)cap);
    W.overflow[scene] = (int)max(0LL, total - cap) + *L.overflow;
}

}  // namespace pdc
