// Device-side building blocks of the B200 contact solver: small 3-vector math,
// the friction-cone functions, and deterministic block reductions.
#pragma once
#include <cooperative_groups.h>
#include <cuda_runtime.h>
#include <stdint.h>

namespace pdc {

// ------------------------------------------------------------ small math
struct d3 { double x, y, z; };
__device__ __forceinline__ d3 mk3(double a, double b, double c) { return d3{a, b, c}; }
__device__ __forceinline__ d3 add3(d3 a, d3 b) { return d3{a.x + b.x, a.y + b.y, a.z + b.z}; }
__device__ __forceinline__ d3 sub3(d3 a, d3 b) { return d3{a.x - b.x, a.y - b.y, a.z - b.z}; }
__device__ __forceinline__ d3 scl3(double s, d3 a) { return d3{s * a.x, s * a.y, s * a.z}; }
__device__ __forceinline__ double dot3(d3 a, d3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
__device__ __forceinline__ d3 cross3(d3 a, d3 b) {
    return d3{a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x};
}
__device__ __forceinline__ d3 ld3(const double* p) { return d3{p[0], p[1], p[2]}; }
__device__ __forceinline__ void st3(double* p, d3 v) { p[0] = v.x; p[1] = v.y; p[2] = v.z; }
__device__ __forceinline__ double dmax(double a, double b) { return (a < b) ? b : a; }  // std::max
__device__ __forceinline__ double dmin(double a, double b) { return (b < a) ? b : a; }  // std::min

// Contact frame R (row-major 3x3, columns n, t1, t2).
struct Frame { double m[9]; };
__device__ __forceinline__ Frame ld_frame(const double* __restrict__ p) {
    Frame f;
#pragma unroll
    for (int i = 0; i < 9; ++i) f.m[i] = __ldg(p + i);
    return f;
}
// R^T v  (world -> contact frame)
__device__ __forceinline__ d3 to_frame(const Frame& R, d3 v) {
    return d3{R.m[0] * v.x + R.m[3] * v.y + R.m[6] * v.z,
              R.m[1] * v.x + R.m[4] * v.y + R.m[7] * v.z,
              R.m[2] * v.x + R.m[5] * v.y + R.m[8] * v.z};
}
// R f  (contact frame -> world)
__device__ __forceinline__ d3 from_frame(const Frame& R, d3 f) {
    return d3{R.m[0] * f.x + R.m[1] * f.y + R.m[2] * f.z,
              R.m[3] * f.x + R.m[4] * f.y + R.m[5] * f.z,
              R.m[6] * f.x + R.m[7] * f.y + R.m[8] * f.z};
}

// ------------------------------------------------ friction cone (a11)
// c(f) = sqrt(ft^2 + p) - mu fn - sqrt(p) - shift, p = 1e-16, shift = 1e-8
// (LorentzCircleConstraint.cpp:5-13, .h:18-19).
#define PDC_PERT 1e-16
#define PDC_SQRT_PERT 1e-8
#define PDC_SHIFT 1e-8
__device__ __forceinline__ double cone_c(double fn, double f1, double f2, double mu) {
    double r = f1 * f1 + f2 * f2 + PDC_PERT;
    return sqrt(r) - mu * fn - PDC_SQRT_PERT - PDC_SHIFT;
}
__device__ __forceinline__ void cone_grad(double f1, double f2, double& g0, double& g1) {
    double r = sqrt(f1 * f1 + f2 * f2 + PDC_PERT);
    g0 = f1 / r;
    g1 = f2 / r;
}
// Hessian (zz^T + p'I) r2^-3/2 with z = (f2, -f1), p' = 1e-6 (:23-35); packed (h00, h01, h11).
__device__ __forceinline__ void cone_hess(double f1, double f2, double& h00, double& h01, double& h11) {
    const double p = 1e-6;
    double r2 = f1 * f1 + f2 * f2 + p;
    double r3 = pow(r2, -1.5);
    h00 = (f2 * f2 + p) * r3;
    h01 = (f2 * -f1) * r3;
    h11 = (f1 * f1 + p) * r3;
}
__device__ __forceinline__ double cone_radius(double fn, double mu) {
    double k = mu * fn + PDC_SQRT_PERT + PDC_SHIFT;
    return sqrt(k * k - PDC_PERT);
}

// ------------------------------------------- deterministic block reductions
// Every thread passes its partial sums; every thread receives the identical
// total (fixed tree: warp shuffle-down to lane 0, per-warp slots, then the same
// tree over the slots in every warp).  `buf` alternates between two halves so a
// single __syncthreads per reduction suffices.
template <int N>
struct BlockReducer {
    double* slots;  // [2][N][32] in shared memory
    int parity;
    __device__ void init(double* s) { slots = s; parity = 0; }
    template <int M>
    __device__ __forceinline__ void sum(double (&v)[M]) {
        static_assert(M <= N, "reduction wider than the slots");
        const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
        double* b = slots + parity * N * 32;
        parity ^= 1;
#pragma unroll
        for (int i = 0; i < M; ++i) {
            double x = v[i];
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) x += __shfl_down_sync(0xffffffffu, x, o);
            if (lane == 0) b[i * 32 + warp] = x;
        }
        __syncthreads();
#pragma unroll
        for (int i = 0; i < M; ++i) {
            double x = (lane < nw) ? b[i * 32 + lane] : 0.0;
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) x += __shfl_down_sync(0xffffffffu, x, o);
            v[i] = __shfl_sync(0xffffffffu, x, 0);
        }
    }
    template <int M>
    __device__ __forceinline__ void max(double (&v)[M]) {
        static_assert(M <= N, "reduction wider than the slots");
        const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
        double* b = slots + parity * N * 32;
        parity ^= 1;
#pragma unroll
        for (int i = 0; i < M; ++i) {
            double x = v[i];
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) x = dmax(x, __shfl_down_sync(0xffffffffu, x, o));
            if (lane == 0) b[i * 32 + warp] = x;
        }
        __syncthreads();
#pragma unroll
        for (int i = 0; i < M; ++i) {
            double x = (lane < nw) ? b[i * 32 + lane] : -INFINITY;
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) x = dmax(x, __shfl_down_sync(0xffffffffu, x, o));
            v[i] = __shfl_sync(0xffffffffu, x, 0);
        }
    }
};

// ------------------------------------------------------------------ teams
// A team is the group of threads that solves one scene: a whole CTA (large
// scenes; __syncthreads, shared-memory reductions) or one warp (small scenes;
// __syncwarp and shuffles only, so a block hosts many independent scenes).
// Both give every member the bitwise-identical result of each reduction.
struct CtaTeam {
    static constexpr int kind = 0;
    static constexpr int spmv_lanes = 1;  // lanes per body in the PCG product
    int rank, size, slot;
    BlockReducer<16> red;
    int* s_int;  // shared: [0] carry, [1..32] warp partials
    __device__ CtaTeam(double* red_smem, int* int_smem) {
        rank = threadIdx.x;
        size = blockDim.x;
        slot = blockIdx.x;
        red.init(red_smem);
        s_int = int_smem;
    }
    __device__ __forceinline__ void sync() { __syncthreads(); }
    template <int N>
    __device__ __forceinline__ void sum(double (&v)[N]) { red.sum(v); }
    template <int N>
    __device__ __forceinline__ void max(double (&v)[N]) { red.max(v); }
    // exclusive scan over n items: put(i, carry0 + prefix)
    template <typename Get, typename Put>
    __device__ void scan(int n, int carry0, Get get, Put put) {
        int* s_carry = s_int;
        int* s_warp = s_int + 1;
        if (rank == 0) *s_carry = carry0;
        __syncthreads();
        const int lane = rank & 31, warp = rank >> 5;
        for (int base = 0; base < n; base += size) {
            const int b = base + rank;
            const int val = (b < n) ? get(b) : 0;
            int x = val;
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                int y = __shfl_up_sync(0xffffffffu, x, o);
                if (lane >= o) x += y;
            }
            if (lane == 31) s_warp[warp] = x;
            __syncthreads();
            if (warp == 0) {
                int w = (lane < (size >> 5)) ? s_warp[lane] : 0;
#pragma unroll
                for (int o = 1; o < 32; o <<= 1) {
                    int y = __shfl_up_sync(0xffffffffu, w, o);
                    if (lane >= o) w += y;
                }
                s_warp[lane] = w;
            }
            __syncthreads();
            const int excl = x - val + (warp ? s_warp[warp - 1] : 0) + *s_carry;
            if (b < n) put(b, excl);
            __syncthreads();
            if (rank == size - 1) *s_carry = excl + val;
            __syncthreads();
        }
    }
};

struct WarpTeam {
    static constexpr int kind = 1;
    static constexpr int spmv_lanes = 1;  // lanes per body in the PCG product
    int rank, size, slot;
    __device__ WarpTeam(int slot_) {
        rank = threadIdx.x & 31;
        size = 32;
        slot = slot_;
    }
    __device__ __forceinline__ void sync() { __syncwarp(); }
    template <int N>
    __device__ __forceinline__ void sum(double (&v)[N]) {
#pragma unroll
        for (int i = 0; i < N; ++i) {
            double x = v[i];
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) x += __shfl_down_sync(0xffffffffu, x, o);
            v[i] = __shfl_sync(0xffffffffu, x, 0);
        }
    }
    template <int N>
    __device__ __forceinline__ void max(double (&v)[N]) {
#pragma unroll
        for (int i = 0; i < N; ++i) {
            double x = v[i];
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) x = dmax(x, __shfl_down_sync(0xffffffffu, x, o));
            v[i] = __shfl_sync(0xffffffffu, x, 0);
        }
    }
    template <typename Get, typename Put>
    __device__ void scan(int n, int carry0, Get get, Put put) {
        int carry = carry0;
        for (int base = 0; base < n; base += 32) {
            const int b = base + rank;
            const int val = (b < n) ? get(b) : 0;
            int x = val;
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                int y = __shfl_up_sync(0xffffffffu, x, o);
                if (rank >= o) x += y;
            }
            if (b < n) put(b, carry + x - val);
            carry += __shfl_sync(0xffffffffu, x, 31);
        }
        __syncwarp();
    }
};

// Grid-wide team for one large scene: a cooperative launch (all blocks
// co-resident), a grid barrier whose wait is bounded (on time-out it raises
// `err` and every block of the launch ends at that barrier), and reductions
// through per-block partials read back in a fixed block order (double-buffered,
// so one barrier per reduction).
struct GridSync {
    unsigned int* count;  // arrivals so far (zeroed before the launch)
    unsigned int* gen;    // generation counter
    int* err;             // set on a barrier time-out; read and cleared by the host
    double* partials;     // [2][gridDim][8]
    int* ipartials;       // [gridDim + 1] block sums for scans
    unsigned long long wait_ns;  // bound on one wait (pdc_config::barrier_timeout_us)
};
#define PDC_BARRIER_SPIN_LIMIT (1LL << 26)

struct GridTeam {
    static constexpr int kind = 2;
    static constexpr int spmv_lanes = 4;  // lanes per body in the PCG product
    int rank, size, slot;
    GridSync G;
    double* s_red;  // shared [8][32] for the in-block stage
    int* s_int;     // shared [33]
    int parity;
    __device__ GridTeam(const GridSync& g, double* red_smem, int* int_smem) {
        rank = blockIdx.x * blockDim.x + threadIdx.x;
        size = gridDim.x * blockDim.x;
        slot = 0;
        G = g;
        s_red = red_smem;
        s_int = int_smem;
        parity = 0;
    }
    // Grid barrier on a counter that only grows (zeroed before the launch): the
    // k-th barrier is passed once the counter reaches k * gridDim.x.  One
    // release-atomic per block to arrive, acquire loads to wait.  A wait longer
    // than G.wait_ns (or PDC_BARRIER_SPIN_LIMIT polls) sets the error flag; a
    // block that sees the flag, its own or another's, ends right there (every
    // thread exits), so no block reads data past a barrier that was not passed:
    // the blocks still running are at most in the phase before it, on data of a
    // barrier they did pass, and they stop at the next barrier.
    unsigned int epoch = 0;
    __device__ void sync() {
        __shared__ int s_stop;
        __syncthreads();
        if (threadIdx.x == 0) {
            volatile int* err = G.err;
            ++epoch;
            int stop = *err;
            if (!stop) {
                const unsigned int target = epoch * gridDim.x;
                unsigned int v;
                __threadfence();
                asm volatile("atom.add.release.gpu.u32 %0, [%1], 1;" : "=r"(v) : "l"(G.count) : "memory");
                ++v;
                long long spins = 0;
                unsigned long long t0 = 0;
                while ((int)(v - target) < 0) {
                    ++spins;
                    if ((spins & 63) == 1) {  // the clock every 64 polls
                        unsigned long long t;
                        asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
                        if (spins == 1) t0 = t;
                        else if (t - t0 > G.wait_ns) spins = PDC_BARRIER_SPIN_LIMIT + 1;
                    }
                    if (spins > PDC_BARRIER_SPIN_LIMIT || *err) {
                        atomicExch(G.err, 1);
                        stop = 1;
                        break;
                    }
                    if (spins > 64) __nanosleep(20);
                    asm volatile("ld.acquire.gpu.u32 %0, [%1];" : "=r"(v) : "l"(G.count) : "memory");
                }
                __threadfence();
            }
            s_stop = stop;
        }
        __syncthreads();
        if (s_stop) asm volatile("exit;");
    }
    template <int N, bool MAX>
    __device__ __forceinline__ void reduce(double (&v)[N]) {
        const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
        double* part = G.partials + (size_t)parity * gridDim.x * 8;
        parity ^= 1;
#pragma unroll
        for (int i = 0; i < N; ++i) {
            double x = v[i];
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) {
                const double y = __shfl_down_sync(0xffffffffu, x, o);
                x = MAX ? dmax(x, y) : x + y;
            }
            if (lane == 0) s_red[i * 32 + warp] = x;
        }
        __syncthreads();
        if (warp == 0) {
#pragma unroll
            for (int i = 0; i < N; ++i) {
                double x = (lane < nw) ? s_red[i * 32 + lane] : (MAX ? -INFINITY : 0.0);
#pragma unroll
                for (int o = 16; o > 0; o >>= 1) {
                    const double y = __shfl_down_sync(0xffffffffu, x, o);
                    x = MAX ? dmax(x, y) : x + y;
                }
                if (lane == 0) part[blockIdx.x * 8 + i] = x;
            }
        }
        sync();
        // every block reduces the partials in the same order: warp 0 strides, then a tree
        if (warp == 0) {
#pragma unroll
            for (int i = 0; i < N; ++i) {
                double x = MAX ? -INFINITY : 0.0;
#pragma unroll 4
                for (int b = lane; b < (int)gridDim.x; b += 32) {
                    const double y = part[b * 8 + i];
                    x = MAX ? dmax(x, y) : x + y;
                }
#pragma unroll
                for (int o = 16; o > 0; o >>= 1) {
                    const double y = __shfl_down_sync(0xffffffffu, x, o);
                    x = MAX ? dmax(x, y) : x + y;
                }
                if (lane == 0) s_red[i * 32] = x;
            }
        }
        __syncthreads();
#pragma unroll
        for (int i = 0; i < N; ++i) v[i] = s_red[i * 32];
        __syncthreads();
    }
    template <int N>
    __device__ __forceinline__ void sum(double (&v)[N]) { reduce<N, false>(v); }
    template <int N>
    __device__ __forceinline__ void max(double (&v)[N]) { reduce<N, true>(v); }
    // exclusive scan over n items (items split into contiguous per-block chunks)
    template <typename Get, typename Put>
    __device__ void scan(int n, int carry0, Get get, Put put) {
        const int chunk = (n + gridDim.x - 1) / gridDim.x;
        const int lo = min(n, (int)blockIdx.x * chunk), hi = min(n, lo + chunk);
        // block sum of the chunk
        int local = 0;
        for (int i = lo + threadIdx.x; i < hi; i += blockDim.x) local += get(i);
        for (int o = 16; o > 0; o >>= 1) local += __shfl_down_sync(0xffffffffu, local, o);
        if ((threadIdx.x & 31) == 0) s_int[1 + (threadIdx.x >> 5)] = local;
        __syncthreads();
        if (threadIdx.x == 0) {
            int t = 0;
            for (int w = 0; w < (int)(blockDim.x >> 5); ++w) t += s_int[1 + w];
            G.ipartials[blockIdx.x] = t;
        }
        sync();
        if (threadIdx.x == 0) {
            int off = carry0;
            for (int b = 0; b < (int)blockIdx.x; ++b) off += G.ipartials[b];
            s_int[0] = off;
        }
        __syncthreads();
        // scan of the chunk, blockDim items at a time
        const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
        for (int base = lo; base < hi; base += blockDim.x) {
            const int i = base + threadIdx.x;
            const int val = (i < hi) ? get(i) : 0;
            int x = val;
            for (int o = 1; o < 32; o <<= 1) {
                const int y = __shfl_up_sync(0xffffffffu, x, o);
                if (lane >= o) x += y;
            }
            if (lane == 31) s_int[1 + warp] = x;
            __syncthreads();
            if (warp == 0) {
                int w = (lane < (int)(blockDim.x >> 5)) ? s_int[1 + lane] : 0;
                for (int o = 1; o < 32; o <<= 1) {
                    const int y = __shfl_up_sync(0xffffffffu, w, o);
                    if (lane >= o) w += y;
                }
                s_int[1 + lane] = w;
            }
            __syncthreads();
            const int excl = x - val + (warp ? s_int[warp] : 0) + s_int[0];
            if (i < hi) put(i, excl);
            __syncthreads();
            if (threadIdx.x == blockDim.x - 1) s_int[0] = excl + val;
            __syncthreads();
        }
        sync();
    }
};

// A thread-block cluster as one team (up to 16 CTAs on neighbouring SMs): the
// hardware cluster barrier (barrier.cluster arrive.release / wait.acquire) is
// about a tenth of the cost of a grid-wide barrier, and reductions exchange the
// per-CTA partials through distributed shared memory.  Every CTA reads the
// partials in the same order, so every thread gets the same bits.
struct ClusterTeam {
    static constexpr int kind = 3;
    static constexpr int spmv_lanes = 4;  // lanes per body in the PCG product
    int rank, size, slot;
    unsigned int crank, csize;
    double* s_red;   // shared [8][32]: in-block stage
    double* s_part;  // shared [2][8]: this CTA's partials, read by every CTA
    int* s_int;      // shared [33]
    int* s_ipart;    // shared [1]: this CTA's block sum in scans
    int parity;
    __device__ ClusterTeam(double* red_smem, double* part_smem, int* int_smem, int* ipart_smem) {
        namespace cg = cooperative_groups;
        cg::cluster_group cl = cg::this_cluster();
        crank = cl.block_rank();
        csize = cl.num_blocks();
        rank = crank * blockDim.x + threadIdx.x;
        size = csize * blockDim.x;
        slot = blockIdx.x / csize;
        s_red = red_smem;
        s_part = part_smem;
        s_int = int_smem;
        s_ipart = ipart_smem;
        parity = 0;
    }
    __device__ __forceinline__ void sync() {
        asm volatile("barrier.cluster.arrive.release.aligned;\n\tbarrier.cluster.wait.acquire.aligned;" ::: "memory");
    }
    template <typename T>
    __device__ __forceinline__ T* remote(T* p, unsigned int r) const {
        return cooperative_groups::this_cluster().map_shared_rank(p, r);
    }
    template <int N, bool MAX>
    __device__ __forceinline__ void reduce(double (&v)[N]) {
        static_assert(N <= 8, "reduction wider than the slots");
        const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
        double* part = s_part + parity * 8;
        parity ^= 1;
#pragma unroll
        for (int i = 0; i < N; ++i) {
            double x = v[i];
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) {
                const double y = __shfl_down_sync(0xffffffffu, x, o);
                x = MAX ? dmax(x, y) : x + y;
            }
            if (lane == 0) s_red[i * 32 + warp] = x;
        }
        __syncthreads();
        if (warp == 0) {
#pragma unroll
            for (int i = 0; i < N; ++i) {
                double x = (lane < nw) ? s_red[i * 32 + lane] : (MAX ? -INFINITY : 0.0);
#pragma unroll
                for (int o = 16; o > 0; o >>= 1) {
                    const double y = __shfl_down_sync(0xffffffffu, x, o);
                    x = MAX ? dmax(x, y) : x + y;
                }
                if (lane == 0) part[i] = x;
            }
        }
        sync();  // partials of every CTA visible cluster-wide
        if (warp == 0) {
#pragma unroll
            for (int i = 0; i < N; ++i) {
                double x = ((unsigned)lane < csize) ? *remote(part + i, lane) : (MAX ? -INFINITY : 0.0);
#pragma unroll
                for (int o = 16; o > 0; o >>= 1) {
                    const double y = __shfl_down_sync(0xffffffffu, x, o);
                    x = MAX ? dmax(x, y) : x + y;
                }
                if (lane == 0) s_red[i * 32] = x;
            }
        }
        __syncthreads();
#pragma unroll
        for (int i = 0; i < N; ++i) v[i] = s_red[i * 32];
        __syncthreads();
    }
    template <int N>
    __device__ __forceinline__ void sum(double (&v)[N]) { reduce<N, false>(v); }
    template <int N>
    __device__ __forceinline__ void max(double (&v)[N]) { reduce<N, true>(v); }
    // exclusive scan over n items (contiguous per-CTA chunks)
    template <typename Get, typename Put>
    __device__ void scan(int n, int carry0, Get get, Put put) {
        const int chunk = (n + (int)csize - 1) / (int)csize;
        const int lo = min(n, (int)crank * chunk), hi = min(n, lo + chunk);
        int local = 0;
        for (int i = lo + threadIdx.x; i < hi; i += blockDim.x) local += get(i);
        for (int o = 16; o > 0; o >>= 1) local += __shfl_down_sync(0xffffffffu, local, o);
        if ((threadIdx.x & 31) == 0) s_int[1 + (threadIdx.x >> 5)] = local;
        __syncthreads();
        if (threadIdx.x == 0) {
            int t = 0;
            for (int w = 0; w < (int)(blockDim.x >> 5); ++w) t += s_int[1 + w];
            *s_ipart = t;
        }
        sync();
        if (threadIdx.x == 0) {
            int off = carry0;
            for (unsigned int b = 0; b < crank; ++b) off += *remote(s_ipart, b);
            s_int[0] = off;
        }
        __syncthreads();
        const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
        for (int base = lo; base < hi; base += blockDim.x) {
            const int i = base + threadIdx.x;
            const int val = (i < hi) ? get(i) : 0;
            int x = val;
            for (int o = 1; o < 32; o <<= 1) {
                const int y = __shfl_up_sync(0xffffffffu, x, o);
                if (lane >= o) x += y;
            }
            if (lane == 31) s_int[1 + warp] = x;
            __syncthreads();
            if (warp == 0) {
                int w = (lane < (int)(blockDim.x >> 5)) ? s_int[1 + lane] : 0;
                for (int o = 1; o < 32; o <<= 1) {
                    const int y = __shfl_up_sync(0xffffffffu, w, o);
                    if (lane >= o) w += y;
                }
                s_int[1 + lane] = w;
            }
            __syncthreads();
            const int excl = x - val + (warp ? s_int[warp] : 0) + s_int[0];
            if (i < hi) put(i, excl);
            __syncthreads();
            if (threadIdx.x == blockDim.x - 1) s_int[0] = excl + val;
            __syncthreads();
        }
        sync();  // every CTA is done reading the block sums
    }
};

// 6x6 symmetric positive definite inverse via Cholesky; input/output packed
// lower triangle, row-major (21 values: (0,0),(1,0),(1,1),(2,0),...).
__device__ __forceinline__ int pk(int r, int c) { return (r >= c) ? (r * (r + 1) / 2 + c) : (c * (c + 1) / 2 + r); }
__device__ inline bool spd6_inverse(const double* A, double* Ainv) {
    double L[21];
#pragma unroll
    for (int j = 0; j < 6; ++j) {
        double d = A[pk(j, j)];
#pragma unroll
        for (int k = 0; k < j; ++k) d -= L[pk(j, k)] * L[pk(j, k)];
        if (!(d > 0.0)) return false;
        double ljj = sqrt(d);
        L[pk(j, j)] = ljj;
#pragma unroll
        for (int i = j + 1; i < 6; ++i) {
            double s = A[pk(i, j)];
#pragma unroll
            for (int k = 0; k < j; ++k) s -= L[pk(i, k)] * L[pk(j, k)];
            L[pk(i, j)] = s / ljj;
        }
    }
    // inverse of L (lower), then Ainv = L^-T L^-1
    double Li[21];
#pragma unroll
    for (int j = 0; j < 6; ++j) {
        Li[pk(j, j)] = 1.0 / L[pk(j, j)];
#pragma unroll
        for (int i = j + 1; i < 6; ++i) {
            double s = 0.0;
#pragma unroll
            for (int k = j; k < i; ++k) s -= L[pk(i, k)] * Li[pk(k, j)];
            Li[pk(i, j)] = s / L[pk(i, i)];
        }
    }
#pragma unroll
    for (int r = 0; r < 6; ++r)
#pragma unroll
        for (int c = 0; c <= r; ++c) {
            double s = 0.0;
#pragma unroll
            for (int k = r; k < 6; ++k) s += Li[pk(k, r)] * Li[pk(k, c)];
            Ainv[pk(r, c)] = s;
        }
    return true;
}

}  // namespace pdc
