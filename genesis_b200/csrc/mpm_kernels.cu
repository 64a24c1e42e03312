// B200-native MLS-MPM substep: counting sort by grid block, fused p2g, grid op, g2p.
//
// Reference path (Genesis, gstaichi kernels):
//   reset_grid_and_grad  mpm_solver.py:540-550   -> folded into k_grid_op (clear after read)
//   compute_F_tmp        mpm_solver.py:261-267   -> k_p2g, registers
//   svd                  mpm_solver.py:269-275   -> k_p2g, registers (svd3.cuh)
//   p2g                  mpm_solver.py:290-389   -> k_p2g (shared-memory tile + float4 red)
//   mpm_grid_op          legacy_coupler.py:352-496 (MPM core) -> k_grid_op over active blocks
//   g2p                  mpm_solver.py:391-449   -> k_g2p (shared-memory velocity tile)
//   _is_state_valid      mpm_solver.py:451-457   -> status bit set in k_g2p, read lazily
//   copy_frame           mpm_solver.py:519-528   -> not needed: state is updated in place
//
// Memory-system design (no tensor cores: MPM is a scatter/gather stencil):
//   * particles live in planar SoA channels, sorted by 4x4x4 grid block every few
//     substeps with a counting sort; each work item ("chunk") is up to P particles of one
//     block, so a warp's loads of any channel are 128-byte coalesced;
//   * p2g accumulates the chunk's 8x8x8-node neighbourhood (the block, its +2 stencil
//     reach and a 1-node drift margin on each side) in shared memory with shared-memory
//     atomics, then flushes only non-empty nodes to the block-major grid with one
//     16-byte vector reduction each, and records which grid blocks became active;
//   * grid op streams the active-block list only (the dense grid is never swept) and
//     re-zeroes mass/momentum behind itself;
//   * g2p stages the same 8x8x8 velocity neighbourhood in shared memory and gathers.
//   Particles that drifted out of their chunk's tile since the last sort take a
//   bounds-checked global-memory path, so stale binning costs speed, never correctness.
#include <cuda_runtime.h>

#include <cstdint>
#include <cstdio>
#include <cstring>
#include <mutex>

#include "../../include/genesis_b200_mpm.h"
#include "constitutive.cuh"
#include "svd3.cuh"

namespace gbm {

// resident threads per SM the register allocation of p2g / g2p2g is sized for: 6 CTAs of 128
// threads at 80 registers (8 B of spills) ran the 500k scene 0.4% faster than 7 at 72 (28 B)
// and 2.2% faster than 8 at 64 (88 B)
#ifndef GBM_P2G_THREADS_PER_SM
#define GBM_P2G_THREADS_PER_SM 768
#endif
// the same for 256- and 512-particle work items: 4 CTAs of 256 threads (64 registers) ran the
// 256-scene batch 1.2% faster than 3 (80 registers); 128-particle items keep 7 CTAs of 128
#ifndef GBM_P2G_THREADS_PER_SM_WIDE
#define GBM_P2G_THREADS_PER_SM_WIDE 1024
#endif
template <int P>
constexpr int kP2GCtasPerSM = (P <= 128 ? GBM_P2G_THREADS_PER_SM : GBM_P2G_THREADS_PER_SM_WIDE) / P;
// unroll factor of the outermost stencil loops (3: fully unrolled, 1: rolled, smaller code)
#ifndef GBM_OUTER_UNROLL
#define GBM_OUTER_UNROLL 3
#endif

// packed float2 arithmetic (sm_100's FFMA2 / FMUL2: two float32 lanes per instruction) in the
// gather and the scatter; each lane is rounded exactly as the scalar form.  GBM_F32X2 for the
// 128-particle work items (bit 0: scatter, bit 1: gather; both measured 2.6% faster on the
// 500k scene, the scatter alone 1.8%)
#ifndef GBM_F32X2
#define GBM_F32X2 3
#endif

constexpr int kOuterUnroll = GBM_OUTER_UNROLL;
// GBM_F32X2_WIDE: the same bits for the 256- and 512-particle work items, whose register
// budget differs (64 registers at 4 CTAs of 256 threads per SM).  With the z channel paired
// with itself in the gather, both packed forms measured faster on the 256-scene batch
// (8.03e9 against 7.91e9 particle-substeps/s with the packed scatter alone)
#ifndef GBM_F32X2_WIDE
#define GBM_F32X2_WIDE 3
#endif
template <int P>
constexpr bool kF32x2Scatter = ((P <= 128 ? GBM_F32X2 : GBM_F32X2_WIDE) & 1) != 0;
template <int P>
constexpr bool kF32x2Gather = ((P <= 128 ? GBM_F32X2 : GBM_F32X2_WIDE) & 2) != 0;
constexpr int BLK = MPM_BLOCK;         // grid block edge
constexpr int BLK3 = BLK * BLK * BLK;  // nodes per block
constexpr int MARGIN = 1;              // drift margin of the shared tile (nodes)
constexpr int TILE = BLK + 2 + 2 * MARGIN;  // 8
constexpr int TN = TILE * TILE * TILE;      // 512
constexpr int SCAN_T = 1024;                // threads of the scan kernels
constexpr int SCAN_ITEMS = 4;               // items per thread
constexpr int SCAN_TILE = SCAN_T * SCAN_ITEMS;
constexpr int MAX_SCAN_TILES = SCAN_T * SCAN_ITEMS;  // single-CTA scan of tile sums
constexpr int64_t MAX_BLOCKS = (int64_t)SCAN_TILE * MAX_SCAN_TILES;

enum Counter {
    CNT_ACTIVE = 0,
    CNT_CHUNKS = 1,
    CNT_STATUS = 2,
    CNT_SORTED = 3,
    CNT_FALLBACK = 4 /* u64 at 4,5 */,
    CNT_DONE = 6,
    CNT_GRID_OPS = 7  // grid ops run on this workspace (the NOISE force field's counter)
};
constexpr int N_COUNTERS = 16;

struct Ws {
    float4* mm;          // grid momentum.xyz + mass, block-major
    float4* gv;          // grid velocity (w unused)
    uint32_t* flag;      // per grid block: 1 if active this substep
    int2* active;        // active block list {instance, packed block coords}
    int* bin_count;      // sort histogram
    int* bin_start;      // exclusive scan of bin_count
    int* chunk_start;    // exclusive scan of chunks per bin
    int* key;            // per particle bin (global block id)
    int* rank;           // per particle rank within its bin
    int4* tile_sums;     // scan scratch
    int4* chunks;        // work items {instance, packed block coords, first slot, end slot}
    float* state_tmp;    // permutation scratch
    uint8_t* mat_tmp;
    uint8_t* pflags_tmp;
    int* gid_tmp;
    float* mu_tmp;
    float* lam_tmp;
    uint32_t* counters;
    uint32_t* inst_status;  // per instance status bits
    int64_t tmp_stride;
};

static inline uint64_t align_up(uint64_t x, uint64_t a) { return (x + a - 1) / a * a; }

constexpr int N_LAYOUT = 19;

struct Layout {
    uint64_t off[N_LAYOUT];
    uint64_t total;
};

static Layout layout_of(const mpm_problem& p) {
    Layout L{};
    const uint64_t nb = (uint64_t)p.n_blocks;
    const uint64_t n = (uint64_t)p.n_particles;
    const uint64_t ntiles = (nb + SCAN_TILE - 1) / SCAN_TILE;
    const uint64_t stride = align_up(n > 0 ? n : 1, 64);
    uint64_t sizes[N_LAYOUT] = {
        nb * BLK3 * 16,            // mm
        nb * BLK3 * 16,            // gv
        nb * 4,                    // flag
        nb * 8,                    // active
        nb * 4,                    // bin_count
        nb * 4,                    // bin_start
        nb * 4,                    // chunk_start
        n * 4,                     // key
        n * 4,                     // rank
        (ntiles + 1) * 16,         // tile_sums
        (uint64_t)p.max_chunks * 16,  // chunks
        stride * MPM_STATE_CH * 4,    // state_tmp
        n,                         // mat_tmp
        n,                         // pflags_tmp
        n * 4,                     // gid_tmp
        n * 4,                     // mu_tmp
        n * 4,                     // lam_tmp
        N_COUNTERS * 4,            // counters
        (uint64_t)p.n_instances * 4,  // per-instance status
    };
    uint64_t o = 0;
    for (int i = 0; i < N_LAYOUT; ++i) {
        L.off[i] = o;
        o = align_up(o + (sizes[i] ? sizes[i] : 1), 256);
    }
    L.total = o;
    return L;
}

static Ws ws_of(const mpm_problem& p, void* base) {
    Layout L = layout_of(p);
    char* b = (char*)base;
    Ws w;
    w.mm = (float4*)(b + L.off[0]);
    w.gv = (float4*)(b + L.off[1]);
    w.flag = (uint32_t*)(b + L.off[2]);
    w.active = (int2*)(b + L.off[3]);
    w.bin_count = (int*)(b + L.off[4]);
    w.bin_start = (int*)(b + L.off[5]);
    w.chunk_start = (int*)(b + L.off[6]);
    w.key = (int*)(b + L.off[7]);
    w.rank = (int*)(b + L.off[8]);
    w.tile_sums = (int4*)(b + L.off[9]);
    w.chunks = (int4*)(b + L.off[10]);
    w.state_tmp = (float*)(b + L.off[11]);
    w.mat_tmp = (uint8_t*)(b + L.off[12]);
    w.pflags_tmp = (uint8_t*)(b + L.off[13]);
    w.gid_tmp = (int*)(b + L.off[14]);
    w.mu_tmp = (float*)(b + L.off[15]);
    w.lam_tmp = (float*)(b + L.off[16]);
    w.counters = (uint32_t*)(b + L.off[17]);
    w.inst_status = (uint32_t*)(b + L.off[18]);
    w.tmp_stride = (int64_t)align_up(p.n_particles > 0 ? p.n_particles : 1, 64);
    return w;
}

// ---------------------------------------------------------------- helpers

__device__ __forceinline__ int find_instance_by_particle(const mpm_instance* inst, int n_inst, int p) {
    int lo = 0, hi = n_inst - 1;
    while (lo < hi) {
        int mid = (lo + hi + 1) >> 1;
        if (__ldg(&inst[mid].p_begin) <= p) lo = mid; else hi = mid - 1;
    }
    return lo;
}

__device__ __forceinline__ int find_instance_by_block(const mpm_instance* inst, int n_inst, int64_t b) {
    int lo = 0, hi = n_inst - 1;
    while (lo < hi) {
        int mid = (lo + hi + 1) >> 1;
        if (__ldg(&inst[mid].blk_base) <= b) lo = mid; else hi = mid - 1;
    }
    return lo;
}

// status bits: one word for the whole problem and one per instance (so a served request
// that went NaN can be evicted without touching the others)
__device__ __forceinline__ void set_status(const Ws& w, int inst, uint32_t bit) {
    atomicOr(&w.counters[CNT_STATUS], bit);
    atomicOr(&w.inst_status[inst], bit);
}

__device__ __forceinline__ float2 dup2(float a) { return make_float2(a, a); }
__device__ __forceinline__ float2 fma2(float2 a, float2 b, float2 c) { return __ffma2_rn(a, b, c); }

// quadratic B-spline weights (mpm_solver.py:350, 397)
__device__ __forceinline__ void bspline(float fx, float* w) {
    const float a = 1.5f - fx;
    const float b = fx - 1.f;
    const float c = fx - 0.5f;
    w[0] = 0.5f * a * a;
    w[1] = 0.75f - b * b;
    w[2] = 0.5f * c * c;
}

// CubeBoundary.impose_pos_vel with restitution 0 (boundaries.py:23-33); velocity part
__device__ __forceinline__ float bc_vel(float pos, float vel, float lo, float hi) {
    if (pos >= hi && vel >= 0.f) return vel * -0.f;
    if (pos <= lo && vel <= 0.f) return vel * -0.f;
    return vel;
}

struct BlockCoord {
    int bx, by, bz;
};

// grid block coordinates packed 10 bits each (nblk < 1024 per axis, checked on the host):
// work items and the active-block list carry them so kernels never divide by nblk
__host__ __device__ __forceinline__ int pack_bc(int bx, int by, int bz) { return bx | (by << 10) | (bz << 20); }
__device__ __forceinline__ BlockCoord unpack_bc(int p) {
    BlockCoord c;
    c.bx = p & 1023;
    c.by = (p >> 10) & 1023;
    c.bz = (p >> 20) & 1023;
    return c;
}
__device__ __forceinline__ int local_block(const mpm_instance& I, int bx, int by, int bz) {
    return (bx * I.nblk[1] + by) * I.nblk[2] + bz;
}

__device__ __forceinline__ BlockCoord block_coord(int lb, const mpm_instance& I) {
    BlockCoord c;
    c.bz = lb % I.nblk[2];
    int t = lb / I.nblk[2];
    c.by = t % I.nblk[1];
    c.bx = t / I.nblk[1];
    return c;
}

__device__ __forceinline__ int64_t node_addr(const mpm_instance& I, int gx, int gy, int gz) {
    const int lb = ((gx >> 2) * I.nblk[1] + (gy >> 2)) * I.nblk[2] + (gz >> 2);
    const int ln = ((gx & 3) * BLK + (gy & 3)) * BLK + (gz & 3);
    return (I.blk_base + lb) * BLK3 + ln;
}

__device__ __forceinline__ void mark_block(Ws& w, int inst, const mpm_instance& I, int bx, int by, int bz) {
    const int lb = (bx * I.nblk[1] + by) * I.nblk[2] + bz;
    uint32_t* f = &w.flag[I.blk_base + lb];
    if (*((volatile uint32_t*)f) == 0u && atomicExch(f, 1u) == 0u) {
        const int i = (int)atomicAdd(&w.counters[CNT_ACTIVE], 1u);
        w.active[i] = make_int2(inst, pack_bc(bx, by, bz));
    }
}

__device__ __forceinline__ bool finite3(float a, float b, float c) {
    return isfinite(a) && isfinite(b) && isfinite(c);
}

// ---------------------------------------------------------------- sort

__global__ void k_sort_keys(mpm_problem prob, const mpm_instance* __restrict__ inst, mpm_particles par, Ws w) {
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= prob.n_particles) return;
    const int k = find_instance_by_particle(inst, prob.n_instances, p);
    const mpm_instance& I = inst[k];
    const int64_t s = par.state_stride;
    const float x0 = par.state[MPM_CH_X * s + p], x1 = par.state[(MPM_CH_X + 1) * s + p],
                x2 = par.state[(MPM_CH_X + 2) * s + p];
    int b[3];
    const float xs[3] = {x0, x1, x2};
#pragma unroll
    for (int d = 0; d < 3; ++d) {
        float f = floorf(xs[d] * I.inv_dx - 0.5f);
        int c = isfinite(f) ? (int)fminf(fmaxf(f - (float)I.lower_cell[d], 0.f), (float)(I.res[d] - 1)) : 0;
        b[d] = min(c >> 2, I.nblk[d] - 1);
    }
    const int lb = (b[0] * I.nblk[1] + b[1]) * I.nblk[2] + b[2];
    const int key = (int)(I.blk_base + lb);
    w.key[p] = key;
    w.rank[p] = atomicAdd(&w.bin_count[key], 1);
}

// Scan of (count, ceil(count/P)) over bins: three phases.
__global__ void k_scan_reduce(int64_t nb, int P, Ws w) {
    __shared__ int s_a[SCAN_T / 32], s_b[SCAN_T / 32];
    const int64_t base = (int64_t)blockIdx.x * SCAN_TILE;
    int a = 0, c = 0;
#pragma unroll
    for (int i = 0; i < SCAN_ITEMS; ++i) {
        int64_t j = base + (int64_t)i * SCAN_T + threadIdx.x;
        if (j < nb) {
            int cnt = w.bin_count[j];
            a += cnt;
            c += (cnt + P - 1) / P;
        }
    }
    for (int o = 16; o > 0; o >>= 1) {
        a += __shfl_down_sync(0xffffffffu, a, o);
        c += __shfl_down_sync(0xffffffffu, c, o);
    }
    if ((threadIdx.x & 31) == 0) {
        s_a[threadIdx.x >> 5] = a;
        s_b[threadIdx.x >> 5] = c;
    }
    __syncthreads();
    if (threadIdx.x < 32) {
        a = s_a[threadIdx.x];
        c = s_b[threadIdx.x];
        for (int o = 16; o > 0; o >>= 1) {
            a += __shfl_down_sync(0xffffffffu, a, o);
            c += __shfl_down_sync(0xffffffffu, c, o);
        }
        if (threadIdx.x == 0) w.tile_sums[blockIdx.x] = make_int4(a, c, 0, 0);
    }
}

// block-wide exclusive scan of (a, c) pairs held one per thread; returns totals
__device__ __forceinline__ int2 block_exscan2(int& a, int& c, int2* s_warp) {
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    int ia = a, ic = c;
    for (int o = 1; o < 32; o <<= 1) {
        int ta = __shfl_up_sync(0xffffffffu, ia, o);
        int tc = __shfl_up_sync(0xffffffffu, ic, o);
        if (lane >= o) {
            ia += ta;
            ic += tc;
        }
    }
    if (lane == 31) s_warp[wid] = make_int2(ia, ic);
    __syncthreads();
    if (wid == 0) {
        const int nw = blockDim.x >> 5;
        int2 v = lane < nw ? s_warp[lane] : make_int2(0, 0);
        int va = v.x, vc = v.y;
        for (int o = 1; o < 32; o <<= 1) {
            int ta = __shfl_up_sync(0xffffffffu, va, o);
            int tc = __shfl_up_sync(0xffffffffu, vc, o);
            if (lane >= o) {
                va += ta;
                vc += tc;
            }
        }
        if (lane < nw) s_warp[lane] = make_int2(va, vc);
    }
    __syncthreads();
    const int2 pre = wid > 0 ? s_warp[wid - 1] : make_int2(0, 0);
    const int2 tot = s_warp[(blockDim.x >> 5) - 1];
    a = pre.x + ia - a;
    c = pre.y + ic - c;
    __syncthreads();
    return tot;
}

__global__ void __launch_bounds__(SCAN_T) k_scan_tiles(int ntiles, Ws w) {
    __shared__ int2 s_warp[32];
    int va[SCAN_ITEMS], vc[SCAN_ITEMS];
    int a = 0, c = 0;
#pragma unroll
    for (int i = 0; i < SCAN_ITEMS; ++i) {
        int j = threadIdx.x * SCAN_ITEMS + i;
        int4 t = j < ntiles ? w.tile_sums[j] : make_int4(0, 0, 0, 0);
        va[i] = t.x;
        vc[i] = t.y;
        a += t.x;
        c += t.y;
    }
    int2 tot = block_exscan2(a, c, s_warp);
#pragma unroll
    for (int i = 0; i < SCAN_ITEMS; ++i) {
        int j = threadIdx.x * SCAN_ITEMS + i;
        if (j < ntiles) w.tile_sums[j] = make_int4(a, c, 0, 0);
        a += va[i];
        c += vc[i];
    }
    if (threadIdx.x == 0) {
        w.counters[CNT_CHUNKS] = (uint32_t)tot.y;
        w.counters[CNT_SORTED] = 1u;
    }
}

__global__ void __launch_bounds__(SCAN_T) k_scan_apply(int64_t nb, int P, Ws w) {
    __shared__ int2 s_warp[32];
    const int64_t base = (int64_t)blockIdx.x * SCAN_TILE + (int64_t)threadIdx.x * SCAN_ITEMS;
    int va[SCAN_ITEMS], vc[SCAN_ITEMS];
    int a = 0, c = 0;
#pragma unroll
    for (int i = 0; i < SCAN_ITEMS; ++i) {
        int64_t j = base + i;
        int cnt = j < nb ? w.bin_count[j] : 0;
        va[i] = cnt;
        vc[i] = (cnt + P - 1) / P;
        a += va[i];
        c += vc[i];
    }
    block_exscan2(a, c, s_warp);
    const int4 t = w.tile_sums[blockIdx.x];
    a += t.x;
    c += t.y;
#pragma unroll
    for (int i = 0; i < SCAN_ITEMS; ++i) {
        int64_t j = base + i;
        if (j < nb) {
            w.bin_start[j] = a;
            w.chunk_start[j] = c;
        }
        a += va[i];
        c += vc[i];
    }
}

__global__ void k_sort_scatter(mpm_problem prob, mpm_particles par, Ws w) {
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= prob.n_particles) return;
    const int dst = w.bin_start[w.key[p]] + w.rank[p];
    const int64_t s = par.state_stride, t = w.tmp_stride;
#pragma unroll 5
    for (int ch = 0; ch < MPM_STATE_CH; ++ch) w.state_tmp[ch * t + dst] = par.state[ch * s + p];
    w.mat_tmp[dst] = par.mat[p];
    w.pflags_tmp[dst] = par.pflags[p];
    w.gid_tmp[dst] = par.gid[p];
    if (par.mu_p) {
        w.mu_tmp[dst] = par.mu_p[p];
        w.lam_tmp[dst] = par.lam_p[p];
    }
}

// Second half of the sort: copy each chunk back from the scratch arrays in an order that
// spreads the chunk's particles over the shared-memory banks.  A particle in in-block cell
// (cx, cy, cz) scatters into tile words whose bank is (4 cx + 8 cy + cz + const) mod 32
// for every stencil node (x-stride 68, y-stride 8), so its bank class
// b = (4 cx + 8 cy + cz) mod 32 (two cells per class) decides its atomics' conflicts: a
// warp costs as many shared-memory wavefronts per atomic as its most repeated class.
//   1. Order: the r-th of the n_b particles of class b gets the key ((2r + 1) / (2 n_b), b)
//      and the chunk is laid out by key, so every class is spread evenly over the chunk
//      and each warp holds about 32 n_b / n of class b (the fewest repeats any split into
//      warps can have, up to rounding).  The position of a particle is the number of
//      smaller keys, summed per class in exact integer arithmetic.
//   2. Deal: inside a full warp, lanes are re-dealt so that the four 8-lane phases of the
//      gather's 16-byte loads (velocity tile slot = b mod 8) each see distinct slots where
//      the warp's classes allow: the warp's particles ranked by (b mod 8, position) go to
//      lane (i mod 4) * 8 + i / 4.
// Also writes gid and the slot map.
template <int P>
__global__ void __launch_bounds__(P) k_sort_interleave(mpm_problem prob, const mpm_instance* __restrict__ inst,
                                                       mpm_particles par, Ws w) {
    __shared__ int cnt[32];
    __shared__ unsigned char s_slot[P];
    const int n_chunks = (int)w.counters[CNT_CHUNKS];
    const int64_t s = par.state_stride, t = w.tmp_stride;
    for (int ci = blockIdx.x; ci < n_chunks; ci += gridDim.x) {
        if (threadIdx.x < 32) cnt[threadIdx.x] = 0;
        __syncthreads();
        const int4 ch = w.chunks[ci];
        const int src = ch.z + threadIdx.x;
        const int n = ch.w - ch.z;
        const bool live = src < ch.w;
        int b = 0, r = 0;
        if (live) {
            const mpm_instance& I = inst[ch.x];
            int c[3];
#pragma unroll
            for (int d = 0; d < 3; ++d) {
                // the cell of k_sort_keys, whose block is this chunk's block
                const float f = floorf(w.state_tmp[(MPM_CH_X + d) * t + src] * I.inv_dx - 0.5f);
                const int cell = isfinite(f) ? (int)fminf(fmaxf(f - (float)I.lower_cell[d], 0.f), (float)(I.res[d] - 1)) : 0;
                c[d] = cell & (BLK - 1);
            }
            b = (4 * c[0] + 8 * c[1] + c[2]) & 31;
            r = atomicAdd(&cnt[b], 1);
        }
        __syncthreads();
        int pos = 0;
        if (live) {
            // #{(b', r') : (2r' + 1) n_b < (2r + 1) n_b', or equal and b' < b}
            const int nb = cnt[b], two_n = 2 * nb;
            const float inv = 1.f / (float)two_n;
#pragma unroll 8
            for (int k = 0; k < 32; ++k) {
                const int nk = cnt[k];
                const int q = (2 * r + 1) * nk - nb;
                int cc;
                if (k == b) {
                    cc = r;
                } else if (q < 0) {
                    cc = 0;
                } else {
                    // q / (2 n_b) to the nearest integer: q < 2^20 and 2 n_b <= 1024, so the
                    // quotient is an integer or at least 1/1024 away from one, far above the
                    // float rounding of q * (1 / (2 n_b)) (below 1e-4 here)
                    const int m = (int)floorf((float)q * inv + 0.5f);
                    if (m * two_n == q)
                        cc = m + ((k < b && m < nk) ? 1 : 0);
                    else
                        cc = m * two_n > q ? m : m + 1;
                    cc = min(cc, nk);
                }
                pos += cc;
            }
            s_slot[pos] = (unsigned char)(b & 7);
        }
        __syncthreads();
        if (live) {
            const int wb = pos & ~31;
            if (wb + 32 <= n) {
                const int sl = b & 7, me = pos & 31;
                int i = 0;
#pragma unroll 8
                for (int j = 0; j < 32; ++j) {
                    const int o = s_slot[wb + j];
                    i += (o < sl || (o == sl && j < me)) ? 1 : 0;
                }
                pos = wb + (i & 3) * 8 + (i >> 2);
            }
            const int dst = ch.z + pos;
#pragma unroll 5
            for (int q = 0; q < MPM_STATE_CH; ++q) par.state[q * s + dst] = w.state_tmp[q * t + src];
            par.mat[dst] = w.mat_tmp[src];
            par.pflags[dst] = w.pflags_tmp[src];
            const int g = w.gid_tmp[src];
            par.gid[dst] = g;
            par.slot[g] = dst;
            if (par.mu_p) {
                par.mu_p[dst] = w.mu_tmp[src];
                par.lam_p[dst] = w.lam_tmp[src];
            }
        }
        __syncthreads();
    }
}

__global__ void k_build_chunks(mpm_problem prob, const mpm_instance* __restrict__ inst, Ws w) {
    const int64_t b = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (b >= prob.n_blocks) return;
    const int cnt = w.bin_count[b];
    if (cnt == 0) return;
    const int P = prob.chunk_particles;
    const int k = find_instance_by_block(inst, prob.n_instances, b);
    const int lb = (int)(b - inst[k].blk_base);
    const BlockCoord bc = block_coord(lb, inst[k]);
    const int pbc = pack_bc(bc.bx, bc.by, bc.bz);
    const int start = w.bin_start[b];
    const int cs = w.chunk_start[b];
    const int nch = (cnt + P - 1) / P;
    for (int j = 0; j < nch; ++j) {
        const int s0 = start + j * P;
        w.chunks[cs + j] = make_int4(k, pbc, s0, min(s0 + P, start + cnt));
    }
}

// ---------------------------------------------------------------- rigid colliders

// MPM_COLLIDER_SDF: distance and geom-frame gradient at geom-frame point l from the sampled
// grid (sdf_func_sdf / sdf_func_grad, utils/sdf_decomp.py:102-276): trilinear inside the grid,
// the distance-to-centre proxy outside it
__device__ __forceinline__ void sdf_sampled(const mpm_collider& c, const float* __restrict__ sdf, float eps,
                                            const float* l, float& sd, float* gl) {
    const int r[3] = {c.sdf_res3[0], c.sdf_res3[1], c.sdf_res3[2]};
    float ps[3], dc[3];
    bool outside = false;
#pragma unroll
    for (int d = 0; d < 3; ++d) {
        const float half = 0.5f * (float)(r[d] - 1);
        ps[d] = c.sdf_scale[d] * (l[d] - c.data[d]) + half;  // data: the grid's centre, geom frame
        dc[d] = ps[d] - half;
        outside = outside || ps[d] >= (float)(r[d] - 1) || ps[d] <= 0.f;
    }
    if (outside) {
        // sdf_func_proxy_sdf / _grad: |p - centre| / cell_size + sdf_max, normalize(p - centre)
        const float d2 = dc[0] * dc[0] + dc[1] * dc[1] + dc[2] * dc[2];
        sd = sqrtf(d2) / c.sdf_cell + c.sdf_max;
        const float inv = rsqrtf(d2 + eps);
#pragma unroll
        for (int d = 0; d < 3; ++d) gl[d] = dc[d] * inv;
        return;
    }
    int b[3];
#pragma unroll
    for (int d = 0; d < 3; ++d) b[d] = min((int)floorf(ps[d]), r[d] - 2);
    const int64_t N = (int64_t)r[0] * r[1] * r[2];
    const float* val = sdf + c.sdf_offset;
    const float* grd = val + N;
    sd = 0.f;
    gl[0] = gl[1] = gl[2] = 0.f;
#pragma unroll
    for (int o = 0; o < 8; ++o) {
        const int cx = b[0] + (o >> 2), cy = b[1] + ((o >> 1) & 1), cz = b[2] + (o & 1);
        const float w = (1.f - fabsf(ps[0] - (float)cx)) * (1.f - fabsf(ps[1] - (float)cy)) * (1.f - fabsf(ps[2] - (float)cz));
        const int64_t idx = ((int64_t)cx * r[1] + cy) * r[2] + cz;
        sd += w * val[idx];
        gl[0] += w * grd[3 * idx + 0];
        gl[1] += w * grd[3 * idx + 1];
        gl[2] += w * grd[3 * idx + 2];
    }
}

// signed distance sd of the geom at p (utils/sdf_decomp.py:75-300), its world gradient g
// (unnormalised for the sphere) and q = p - the geom's origin
__device__ __forceinline__ void sdf_grad(const mpm_collider& c, const float* __restrict__ sdf, float eps,
                                         const float* p, float& sd, float* g, float* q) {
    q[0] = p[0] - c.pos[0];
    q[1] = p[1] - c.pos[1];
    q[2] = p[2] - c.pos[2];
    if (c.kind == MPM_COLLIDER_SPHERE) {
        sd = sqrtf(q[0] * q[0] + q[1] * q[1] + q[2] * q[2]) - c.data[0];
        g[0] = q[0];
        g[1] = q[1];
        g[2] = q[2];
    } else {
        float l[3], gl[3];  // geom-frame point and gradient
#pragma unroll
        for (int i = 0; i < 3; ++i) l[i] = c.rot[0 * 3 + i] * q[0] + c.rot[1 * 3 + i] * q[1] + c.rot[2 * 3 + i] * q[2];
        if (c.kind == MPM_COLLIDER_PLANE) {
            sd = l[0] * c.data[0] + l[1] * c.data[1] + l[2] * c.data[2];
            gl[0] = c.data[0];
            gl[1] = c.data[1];
            gl[2] = c.data[2];
        } else if (c.kind == MPM_COLLIDER_SDF) {
            sdf_sampled(c, sdf, eps, l, sd, gl);
        } else {
            float d[3], o[3];
#pragma unroll
            for (int i = 0; i < 3; ++i) {
                d[i] = fabsf(l[i]) - c.data[i];
                o[i] = fmaxf(d[i], 0.f);
            }
            const float out = sqrtf(o[0] * o[0] + o[1] * o[1] + o[2] * o[2]);
            const float dm = fmaxf(d[0], fmaxf(d[1], d[2]));
            sd = out + fminf(dm, 0.f);
            if (out > 0.f) {
#pragma unroll
                for (int i = 0; i < 3; ++i) gl[i] = copysignf(o[i], l[i]) / out;
            } else {
                const int a = (d[0] >= d[1] && d[0] >= d[2]) ? 0 : (d[1] >= d[2] ? 1 : 2);
#pragma unroll
                for (int i = 0; i < 3; ++i) gl[i] = (i == a) ? copysignf(1.f, l[i]) : 0.f;
            }
        }
#pragma unroll
        for (int i = 0; i < 3; ++i) g[i] = c.rot[i * 3 + 0] * gl[0] + c.rot[i * 3 + 1] * gl[1] + c.rot[i * 3 + 2] * gl[2];
    }
}

// unit outward normal (sdf_func_normal_world); the sphere's gradient is q / sqrt(|q|^2 + eps)
// before the normalisation, as ti_normalize(q, EPS) gives it
__device__ __forceinline__ void unit_normal(const mpm_collider& c, float eps, float* g, float* n) {
    if (c.kind == MPM_COLLIDER_SPHERE) {
        const float inv = rsqrtf(g[0] * g[0] + g[1] * g[1] + g[2] * g[2] + eps);
        g[0] *= inv;
        g[1] *= inv;
        g[2] *= inv;
    }
    const float ninv = rsqrtf(g[0] * g[0] + g[1] * g[1] + g[2] * g[2] + eps);
    n[0] = g[0] * ninv;
    n[1] = g[1] * ninv;
    n[2] = g[2] * ninv;
}

__device__ __forceinline__ void collider_normal(const mpm_collider& c, const float* __restrict__ sdf, float eps,
                                                const float* p, float* n) {
    float sd, g[3], q[3];
    sdf_grad(c, sdf, eps, p, sd, g, q);
    unit_normal(c, eps, g, n);
}

// legacy_coupler.py:297-341 (_func_collide_in_rigid_geom) for a point at q from the collider
// origin with outward normal n and influence infl: v relative to the collider's velocity at
// the point loses its inward normal part (restitution) and is slowed tangentially
// (friction); the momentum change goes to fout[6] as force and torque about the origin
__device__ __forceinline__ void rigid_respond(const mpm_collider& c, float eps, float dt, float mass, const float* q,
                                              const float* n, float infl, float* v, float* fout) {
    // velocity of the collider at p (rigid_solver_decomp.py:3413-3419)
    const float vr[3] = {c.lin_vel[0] + c.ang_vel[1] * q[2] - c.ang_vel[2] * q[1],
                         c.lin_vel[1] + c.ang_vel[2] * q[0] - c.ang_vel[0] * q[2],
                         c.lin_vel[2] + c.ang_vel[0] * q[1] - c.ang_vel[1] * q[0]};
    const float rv[3] = {v[0] - vr[0], v[1] - vr[1], v[2] - vr[2]};
    const float rn = rv[0] * n[0] + rv[1] * n[1] + rv[2] * n[2];
    if (!(rn < 0.f)) return;
    float rt[3] = {rv[0] - rn * n[0], rv[1] - rn * n[1], rv[2] - rn * n[2]};
    const float rtn = sqrtf(rt[0] * rt[0] + rt[1] * rt[1] + rt[2] * rt[2] + eps);
    const float sc = fmaxf(0.f, rtn + rn * c.friction) / rtn;
    float dv[3];
#pragma unroll
    for (int i = 0; i < 3; ++i) {
        const float rnew = rt[i] * sc - n[i] * rn * c.restitution;
        const float nvi = vr[i] + rnew * infl + rv[i] * (1.f - infl);
        dv[i] = nvi - v[i];
        v[i] = nvi;
    }
    if (fout) {
        const float f[3] = {-mass * dv[0] / dt, -mass * dv[1] / dt, -mass * dv[2] / dt};
        atomicAdd(&fout[0], f[0]);
        atomicAdd(&fout[1], f[1]);
        atomicAdd(&fout[2], f[2]);
        atomicAdd(&fout[3], q[1] * f[2] - q[2] * f[1]);
        atomicAdd(&fout[4], q[2] * f[0] - q[0] * f[2]);
        atomicAdd(&fout[5], q[0] * f[1] - q[1] * f[0]);
    }
}

// the grid op's coupling of one node (legacy_coupler.py:166-343): influence
// min(exp(-sd / softness), 1), acting above 0.1
__device__ __forceinline__ void collide_rigid(const mpm_collider& c, const float* __restrict__ sdf, float eps, float dt,
                                              float mass, const float* p, float* v, float* fout) {
    float sd, g[3], q[3], n[3];
    sdf_grad(c, sdf, eps, p, sd, g, q);
    const float influence = fminf(expf(-sd / fmaxf(1e-10f, c.softness)), 1.f);
    if (!(influence > 0.1f)) return;
    unit_normal(c, eps, g, n);
    rigid_respond(c, eps, dt, mass, q, n, influence, v, fout);
}

// ---------------------------------------------------------------- tool entities
// engine/entities/tool_entity/mesh.py:80-176 (Tool.collide), coupled by
// legacy_coupler.py:346-350 before the rigid geoms.

// E = exp([w] dt) (Rodrigues), the rotation of one substep at angular velocity w; the
// quaternion product of tool_entity.py:183-186 and the rigid colliders' motion are this
// rotation applied in the world frame (E R)
__device__ __forceinline__ void rot_step(const float* w, float dt, float* E) {
    const float wx = w[0] * dt, wy = w[1] * dt, wz = w[2] * dt;
    const float th = sqrtf(wx * wx + wy * wy + wz * wz);
    if (!(th > 0.f)) {
#pragma unroll
        for (int k = 0; k < 9; ++k) E[k] = (k % 4 == 0) ? 1.f : 0.f;
        return;
    }
    const float kx = wx / th, ky = wy / th, kz = wz / th, s = sinf(th), c = cosf(th), t = 1.f - c;
    E[0] = c + t * kx * kx;
    E[1] = t * kx * ky - s * kz;
    E[2] = t * kx * kz + s * ky;
    E[3] = t * kx * ky + s * kz;
    E[4] = c + t * ky * ky;
    E[5] = t * ky * kz - s * kx;
    E[6] = t * kx * kz - s * ky;
    E[7] = t * ky * kz + s * kx;
    E[8] = c + t * kz * kz;
}

// mesh.py:89-104: trilinear sample of the voxel grid at voxel coordinate pv; 1 outside it
__device__ __forceinline__ float tool_sdf_at(const float* __restrict__ vox, int res, const float* pv) {
    const float f0 = floorf(pv[0]), f1 = floorf(pv[1]), f2 = floorf(pv[2]);
    if (!(f0 >= 0.f && f1 >= 0.f && f2 >= 0.f && f0 < (float)(res - 1) && f1 < (float)(res - 1) &&
          f2 < (float)(res - 1)))
        return 1.f;
    const int b0 = (int)f0, b1 = (int)f1, b2 = (int)f2;
    float sd = 0.f;
#pragma unroll
    for (int o = 0; o < 8; ++o) {
        const int i = o >> 2, j = (o >> 1) & 1, k = o & 1;
        const float w = (1.f - fabsf(pv[0] - (float)(b0 + i))) * (1.f - fabsf(pv[1] - (float)(b1 + j))) *
                        (1.f - fabsf(pv[2] - (float)(b2 + k)));
        sd += w * vox[((int64_t)(b0 + i) * res + (b1 + j)) * res + (b2 + k)];
    }
    return sd;
}

// Tool.collide for a grid node at p with velocity v (mesh.py:147-176)
__device__ __forceinline__ void collide_tool(const mpm_collider& c, const float* __restrict__ sdf_voxels, float eps,
                                             float dt, const float* p, float* v) {
    if (!sdf_voxels || c.sdf_res < 2) return;
    const float q[3] = {p[0] - c.pos[0], p[1] - c.pos[1], p[2] - c.pos[2]};
    const float half = 0.5f * (float)(c.sdf_res - 1);
    float pv[3];
#pragma unroll
    for (int i = 0; i < 3; ++i)
        pv[i] = c.sdf_scale[i] * (c.rot[0 * 3 + i] * q[0] + c.rot[1 * 3 + i] * q[1] + c.rot[2 * 3 + i] * q[2]) + half;
    const float* vox = sdf_voxels + c.sdf_offset;
    const float sd = tool_sdf_at(vox, c.sdf_res, pv);
    const float influence = fminf(expf(-sd / fmaxf(eps, c.softness)), 1.f);
    if (!(sd <= 0.f || influence > 0.1f)) return;
    // vel_collider (mesh.py:139-145): where the body point at p is one substep later, minus p,
    // over dt.  Written as ((E - I) q + dpos) / dt with (E - I) q = sin(th) k x q +
    // 2 sin^2(th / 2) k x (k x q), so the difference of the two poses loses no digits
    float vc[3];
    {
        const float wx = c.ang_vel[0] * dt, wy = c.ang_vel[1] * dt, wz = c.ang_vel[2] * dt;
        const float th = sqrtf(wx * wx + wy * wy + wz * wz);
        float d[3] = {0.f, 0.f, 0.f};
        if (th > 0.f) {
            const float k[3] = {wx / th, wy / th, wz / th};
            const float kq[3] = {k[1] * q[2] - k[2] * q[1], k[2] * q[0] - k[0] * q[2], k[0] * q[1] - k[1] * q[0]};
            const float kkq[3] = {k[1] * kq[2] - k[2] * kq[1], k[2] * kq[0] - k[0] * kq[2], k[0] * kq[1] - k[1] * kq[0]};
            const float sh = sinf(0.5f * th), s = sinf(th), t = 2.f * sh * sh;
#pragma unroll
            for (int i = 0; i < 3; ++i) d[i] = s * kq[i] + t * kkq[i];
        }
        float dz = c.lin_vel[2] * dt;
        if (c.pos[2] + dz < c.floor) dz = c.floor - c.pos[2];  // FloorBoundary.impose_pos of the origin
        vc[0] = (d[0] + c.lin_vel[0] * dt) / dt;
        vc[1] = (d[1] + c.lin_vel[1] * dt) / dt;
        vc[2] = (d[2] + dz) / dt;
    }
    const float rv[3] = {v[0] - vc[0], v[1] - vc[1], v[2] - vc[2]};
    // normal (mesh.py:107-137): central differences of 1e-2 voxel, normalised, mapped to the
    // mesh frame by the inverse voxel scale and to the world by the pose, normalised again
    float nv[3];
#pragma unroll
    for (int i = 0; i < 3; ++i) {
        float a[3] = {pv[0], pv[1], pv[2]}, b[3] = {pv[0], pv[1], pv[2]};
        a[i] += 1e-2f;
        b[i] -= 1e-2f;
        nv[i] = (tool_sdf_at(vox, c.sdf_res, a) - tool_sdf_at(vox, c.sdf_res, b)) / 2e-2f;
    }
    float inv = rsqrtf(nv[0] * nv[0] + nv[1] * nv[1] + nv[2] * nv[2] + eps);
    const float nm[3] = {nv[0] * inv / c.sdf_scale[0], nv[1] * inv / c.sdf_scale[1], nv[2] * inv / c.sdf_scale[2]};
    float n[3];
#pragma unroll
    for (int i = 0; i < 3; ++i) n[i] = c.rot[i * 3 + 0] * nm[0] + c.rot[i * 3 + 1] * nm[1] + c.rot[i * 3 + 2] * nm[2];
    inv = rsqrtf(n[0] * n[0] + n[1] * n[1] + n[2] * n[2] + eps);
    n[0] *= inv;
    n[1] *= inv;
    n[2] *= inv;
    const float rn = rv[0] * n[0] + rv[1] * n[1] + rv[2] * n[2];
    if (!(rn < 0.f)) return;
    const float rt[3] = {rv[0] - rn * n[0], rv[1] - rn * n[1], rv[2] - rn * n[2]};
    const float rtn = sqrtf(rt[0] * rt[0] + rt[1] * rt[1] + rt[2] * rt[2] + eps);
    const float sc = fmaxf(0.f, rtn + rn * c.friction) / rtn;
#pragma unroll
    for (int i = 0; i < 3; ++i) v[i] = vc[i] + rt[i] * sc * influence + rv[i] * (1.f - influence);
}

// ---------------------------------------------------------------- p2g

struct P2GArgs {
    mpm_problem prob;
    const mpm_instance* inst;
    const mpm_material* mats;
    mpm_particles par;
    Ws w;
    const mpm_collider* cols;  // CPIC variants only
    int n_cols;
    float* cforce;
    const float* sdf_voxels;   // sampled grids of MPM_COLLIDER_TOOL / _SDF colliders
};

// Shared tile in int32 fixed point.  On sm_100 shared-memory float atomicAdd is not a
// native operation (it measures 3.3x slower than int32 even without conflicts, 4x with
// the random conflicts of a stencil scatter) while int32 shared atomics are; the tile is
// therefore accumulated as integers.  Each chunk picks, per channel, a power-of-two scale
// s with max(n, 256) * b * s < 2^30, where n is the number of particles in the chunk and b
// bounds |contribution| of any of them to any node (w <= 1, |off - fx| <= 1.5): no node
// sum can overflow, every contribution is below 2^22 (so round-to-nearest is one fused
// multiply-add of the weight with 1.5 * 2^23), and the quantisation step is 2^-22 of the
// chunk's largest contribution, on a par with float32 accumulation.  The tile uses an
// x-stride of 68 words so the banks of a 4x4x4 block's nodes spread over all 32 banks.
constexpr int TXS = TILE * TILE + 4;       // skewed x-stride of the shared tile (words)
constexpr int TWORDS = TILE * TXS;         // words per channel (544)

__device__ __forceinline__ int tidx(int x, int y, int z) { return x * TXS + y * TILE + z; }

__device__ __forceinline__ float warp_max(float v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v = fmaxf(v, __shfl_xor_sync(0xffffffffu, v, o));
    return v;
}

// round-to-nearest integer of the exact product a * b for |a * b| < 2^22: the fused add of
// 1.5 * 2^23 leaves it in the low mantissa bits (one rounding, one instruction)
__device__ __forceinline__ int fix_mul(float a, float b) {
    return __float_as_int(__fmaf_rn(a, b, 12582912.0f)) - 0x4B400000;
}

struct Tile {
    int t[4][TWORDS];  // momentum x, y, z, mass
    float red[2][32];  // per-warp payload bounds
    int wcnt[32];      // per-warp in-tile particle counts
    int wreach[32];    // per-warp stencil reach into the neighbour blocks (6 bits)
};

// Grid velocities of the 8^3 tile, float4 per node, laid out like the atomic tile
// (x-stride 68 nodes, y-stride 8): the 16-byte slot of a lane's every stencil node is then
// (4 cx + cz + const) mod 8, i.e. its bank class mod 8, which the sort's lane deal keeps
// distinct within each 8-lane phase of a 16-byte load.
constexpr int VYS = TILE;           // y-stride (nodes)
constexpr int VXS = TXS;            // x-stride (68 nodes)
static_assert(VXS == TXS && VYS == TILE, "the velocity tile shares the scatter tile's node index");
__device__ __forceinline__ int vidx(int x, int y, int z) { return x * VXS + y * VYS + z; }

struct VelTile {
    float4 v[TILE * VXS];
};

// Per-thread scatter payload of one particle: mass * v + affine (off - fx) dx = q + A off.
struct Payload {
    float q[3], A[9], fx[3];
    float mass, bq;
    int base[3];
    bool live, in_tile;
    int slot, gid;  // CPIC variants only (-1: no particle)
};

// element i of a 3-array without dynamic indexing (keeps it in registers in rolled loops)
__device__ __forceinline__ float sel3(const float* w, int i) { return i == 0 ? w[0] : (i == 1 ? w[1] : w[2]); }

__device__ __forceinline__ void locate(const mpm_instance& I, const float* x, int* base, float* fx) {
#pragma unroll
    for (int d = 0; d < 3; ++d) {
        const float xi = x[d] * I.inv_dx;
        const float bf = floorf(xi - 0.5f);
        base[d] = (int)fminf(fmaxf(bf, -1e8f), 1e8f) - I.lower_cell[d];
        fx[d] = xi - bf;
    }
}

__device__ __forceinline__ bool tile_contains(const int* base, int ox, int oy, int oz) {
    const int lx = base[0] - ox, ly = base[1] - oy, lz = base[2] - oz;
    return lx >= 0 && ly >= 0 && lz >= 0 && lx <= TILE - 3 && ly <= TILE - 3 && lz <= TILE - 3;
}

// per-thread shared-memory parking space for x, v, C (15 words, stride P: conflict-free);
// 512-thread CTAs keep them in registers (their tiles leave no room under 48 KB)
template <int P>
constexpr bool kStash = P <= 256;
template <int P>
struct Stash {
    float s[15][kStash<P> ? P : 1];
};

// compute_F_tmp + svd + return mapping + stress (mpm_solver.py:261-345) for slot p with
// velocity v and affine C; writes F and Jp of the next frame and fills the scatter payload
// for position x.
// MUSCLE: compiled with the Muscle actuation term (a separate instantiation, so problems
// without muscles pay no registers for it)
template <int P, bool MUSCLE>
__device__ __forceinline__ void particle_update(const mpm_instance& I, const mpm_material* __restrict__ mats,
                                                const mpm_particles& par, int p, const float* x_in,
                                                const float* v_in, const float* C_in, int ox, int oy, int oz,
                                                Payload& o, const Ws& w, int inst, Stash<P>& sh) {
    const int64_t st = par.state_stride;
    float* __restrict__ S = par.state;
    float F[9];
#pragma unroll
    for (int k = 0; k < 9; ++k) F[k] = S[(MPM_CH_F + k) * st + p];
    const float Jp = S[MPM_CH_JP * st + p];
    const mpm_material m = mats[I.mat_base + par.mat[p]];
    float mu = m.mu, lam = m.lam;
    if (par.mu_p) {
        // an inviscid Liquid keeps mu = 0 whatever its per-particle E (liquid.py:47-48)
        mu = (m.kind == MPM_MAT_LIQUID && m.mu == 0.f) ? 0.f : par.mu_p[p];
        lam = par.lam_p[p];
    }
    // compute_F_tmp: (I + dt C) F   (mpm_solver.py:264-266)
    float Ft[9];
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = 0; j < 3; ++j) {
            float acc = F[i * 3 + j];
#pragma unroll
            for (int k = 0; k < 3; ++k) acc += I.dt * C_in[i * 3 + k] * F[k * 3 + j];
            Ft[i * 3 + j] = acc;
        }
    // x, v and C are needed again only for the scatter payload: park them in shared
    // memory across the SVD and return mapping, where register pressure peaks
    // (volatile, so the compiler cannot keep them in registers instead)
    float x[3], v[3], C[9];
    if constexpr (kStash<P>) {
        volatile float* sv = &sh.s[0][threadIdx.x];
#pragma unroll
        for (int k = 0; k < 3; ++k) {
            sv[k * P] = x_in[k];
            sv[(3 + k) * P] = v_in[k];
        }
#pragma unroll
        for (int k = 0; k < 9; ++k) sv[(6 + k) * P] = C_in[k];
    }
    float U[9], Sg[3], V[9];
    svd3(Ft, U, Sg, V, needs_uv(m, mu));
    const float J = Sg[0] * (Sg[1] * Sg[2]);
    float Fn[9], stress[9], Jpn;
    constitutive(m, mu, lam, I.eps, J, Ft, U, Sg, V, Jp, Fn, Jpn, stress);
    if (MUSCLE && (m.flags & MPM_MATF_MUSCLE) && par.actu) {
        // muscle.py:57-65: + stiffness * actu * F_tmp d d^T F_tmp^T; a Muscle is an Elastic,
        // whose F_new is F_tmp, so Fn stands in for F_tmp here
        const int g = par.gid[p];
        const float dd[3] = {par.muscle_dir[3 * g], par.muscle_dir[3 * g + 1], par.muscle_dir[3 * g + 2]};
        const float k = m.muscle_stiffness * par.actu[g];
        float fd[3];
#pragma unroll
        for (int i = 0; i < 3; ++i) fd[i] = Fn[i * 3] * dd[0] + Fn[i * 3 + 1] * dd[1] + Fn[i * 3 + 2] * dd[2];
#pragma unroll
        for (int i = 0; i < 3; ++i)
#pragma unroll
            for (int j = 0; j < 3; ++j) stress[i * 3 + j] += k * fd[i] * fd[j];
    }
#pragma unroll
    for (int k = 0; k < 9; ++k) S[(MPM_CH_F + k) * st + p] = Fn[k];
    S[MPM_CH_JP * st + p] = Jpn;
    if constexpr (kStash<P>) {
        volatile float* sv = &sh.s[0][threadIdx.x];
#pragma unroll
        for (int k = 0; k < 3; ++k) {
            x[k] = sv[k * P];
            v[k] = sv[(3 + k) * P];
        }
#pragma unroll
        for (int k = 0; k < 9; ++k) C[k] = sv[(6 + k) * P];
    } else {
#pragma unroll
        for (int k = 0; k < 3; ++k) {
            x[k] = x_in[k];
            v[k] = v_in[k];
        }
#pragma unroll
        for (int k = 0; k < 9; ++k) C[k] = C_in[k];
    }
    // affine = stress * (-dt vol 4 inv_dx^2) + mass C (mpm_solver.py:344-345)
    o.mass = m.mass;
    float A[9];
#pragma unroll
    for (int k = 0; k < 9; ++k) A[k] = I.stress_scale * stress[k] + o.mass * C[k];
    o.live = false;
    o.in_tile = false;
    o.bq = 0.f;
    if (finite3(x[0], x[1], x[2])) {
        o.live = true;
        locate(I, x, o.base, o.fx);
        const float dx = I.dx;
#pragma unroll
        for (int i = 0; i < 3; ++i) {
            o.q[i] = o.mass * v[i] - (A[i * 3 + 0] * o.fx[0] + A[i * 3 + 1] * o.fx[1] + A[i * 3 + 2] * o.fx[2]) * dx;
            const float b =
                fabsf(o.mass * v[i]) + 1.5f * dx * (fabsf(A[i * 3 + 0]) + fabsf(A[i * 3 + 1]) + fabsf(A[i * 3 + 2]));
            o.bq = fmaxf(o.bq, b);
        }
        // fmaxf drops NaN, so test the payload itself: a NaN or Inf must take the float path
        // (where it propagates into the grid as in the reference), never the fixed-point tile
        float chk = o.q[0] + o.q[1] + o.q[2] + o.mass;
#pragma unroll
        for (int k = 0; k < 9; ++k) {
            o.A[k] = A[k] * dx;
            chk += o.A[k];
        }
        o.in_tile = tile_contains(o.base, ox, oy, oz) && isfinite(o.bq) && isfinite(chk);
    } else {
        set_status(w, inst, MPM_STATUS_NAN);
    }
}

// ---------------------------------------------------------------- CPIC
// mpm_solver.py:357-379, 412-427 and legacy_coupler.py:498-525, against the colliders.

// coupler.preprocess: the particle (API id g, at x) takes each collider's normal at x unless it
// points against the one it remembers, i.e. unless it has crossed the collider
__device__ __forceinline__ void cpic_update_normals(const P2GArgs& a, int inst, const mpm_instance& I, int g,
                                                    const float* x) {
    const int64_t st = a.par.state_stride;
    for (int k = 0; k < a.n_cols; ++k) {
        const mpm_collider& c = a.cols[k];
        if (c.instance != inst || c.kind == MPM_COLLIDER_TOOL) continue;  // CPIC: rigid geoms only
        float n[3];
        collider_normal(c, a.sdf_voxels, I.eps, x, n);
        float* o = a.par.cpic_normal + (int64_t)(3 * k) * st + g;
        if (n[0] * o[0] + n[1] * o[st] + n[2] * o[2 * st] >= 0.f) {
            o[0] = n[0];
            o[st] = n[1];
            o[2 * st] = n[2];
        }
    }
}

// 1 + the first collider whose normal at grid node (gx, gy, gz) points against the one
// particle g remembers (it separates them), or 0
__device__ __forceinline__ uint32_t cpic_separating(const P2GArgs& a, int inst, const mpm_instance& I, int g, int gx,
                                                    int gy, int gz) {
    const float pos[3] = {(float)(gx + I.lower_cell[0]) * I.dx, (float)(gy + I.lower_cell[1]) * I.dx,
                          (float)(gz + I.lower_cell[2]) * I.dx};
    const int64_t st = a.par.state_stride;
    for (int k = 0; k < a.n_cols; ++k) {
        const mpm_collider& c = a.cols[k];
        if (c.instance != inst || c.kind == MPM_COLLIDER_TOOL) continue;  // CPIC: rigid geoms only
        float n[3];
        collider_normal(c, a.sdf_voxels, I.eps, pos, n);
        const float* o = a.par.cpic_normal + (int64_t)(3 * k) * st + g;
        if (n[0] * o[0] + n[1] * o[st] + n[2] * o[2 * st] < 0.f) return (uint32_t)(k + 1);
    }
    return 0u;
}

// the separated nodes' byte codes of one particle (slot p) for the g2p that follows; byte 27
// flags that there is at least one
__device__ __forceinline__ void cpic_store(const P2GArgs& a, int p, uint32_t* sw) {
    const int64_t st = a.par.state_stride;
    if (sw[0] | sw[1] | sw[2] | sw[3] | sw[4] | sw[5] | sw[6]) sw[6] |= 1u << 24;
#pragma unroll
    for (int q = 0; q < 7; ++q) a.par.cpic_sep[q * st + p] = sw[q];
}

// g2p of the separated nodes: instead of the grid velocity, the particle's own velocity after
// the rigid response along the normal it remembers (influence 1, mass m w / 1e3; the
// reaction goes to the collider's force)
__device__ __forceinline__ void cpic_correct(const P2GArgs& a, const VelTile* VT, const Ws& w, const mpm_instance& I,
                                             int p, const float* x, const int* base, const float* fx, const float* wx,
                                             const float* wy, const float* wz, bool tile, int ox, int oy, int oz,
                                             float* nv, float* nC) {
    const int64_t st = a.par.state_stride;
    const uint32_t w6 = a.par.cpic_sep[6 * st + p];
    if (!(w6 >> 24)) return;
    uint32_t sw[7];
#pragma unroll
    for (int q = 0; q < 6; ++q) sw[q] = a.par.cpic_sep[q * st + p];
    sw[6] = w6;
    const int g = a.par.gid[p];
    const float mass = a.mats[I.mat_base + a.par.mat[p]].mass;
    const float v0[3] = {a.par.state[(MPM_CH_V + 0) * st + p], a.par.state[(MPM_CH_V + 1) * st + p],
                         a.par.state[(MPM_CH_V + 2) * st + p]};
#pragma unroll 1
    for (int nidx = 0; nidx < 27; ++nidx) {
        const uint32_t sg = (sw[nidx >> 2] >> (8 * (nidx & 3))) & 255u;
        if (!sg) continue;
        const int i = nidx / 9, j = (nidx / 3) % 3, k = nidx % 3;
        const int gx = base[0] + i, gy = base[1] + j, gz = base[2] + k;
        float4 gvn;
        if (tile) {
            gvn = VT->v[vidx(gx - ox, gy - oy, gz - oz)];
        } else {
            if (gx < 0 || gy < 0 || gz < 0 || gx >= I.res[0] || gy >= I.res[1] || gz >= I.res[2]) continue;
            gvn = w.gv[node_addr(I, gx, gy, gz)];
        }
        const mpm_collider& c = a.cols[sg - 1];
        const float wt = sel3(wx, i) * sel3(wy, j) * sel3(wz, k);
        float vs[3] = {v0[0], v0[1], v0[2]};
        const float q[3] = {x[0] - c.pos[0], x[1] - c.pos[1], x[2] - c.pos[2]};
        const float* on = a.par.cpic_normal + (int64_t)(3 * (sg - 1)) * st + g;
        const float n[3] = {on[0], on[st], on[2 * st]};
        rigid_respond(c, I.eps, I.dt, mass * wt / 1e3f, q, n, 1.f, vs, a.cforce ? a.cforce + 6 * (sg - 1) : nullptr);
        const float dv[3] = {vs[0] - gvn.x, vs[1] - gvn.y, vs[2] - gvn.z};
        const float off[3] = {(float)i - fx[0], (float)j - fx[1], (float)k - fx[2]};
#pragma unroll
        for (int d = 0; d < 3; ++d) {
            nv[d] += wt * dv[d];
#pragma unroll
            for (int e = 0; e < 3; ++e) nC[d * 3 + e] += I.c_scale * wt * dv[d] * off[e];
        }
    }
}

// Tile node n of the 8^3 tile whose origin is (4b - 1) per axis lies in grid block b + db
// (db in {-1, 0, 1}) at in-block offset (t + 3) & 3.  These depend only on n, so each
// thread packs them once for the nodes it owns:
//   bits 0-5 in-block node index, 6-10 neighbour id (dbx + 1) 9 + (dby + 1) 3 + (dbz + 1),
//   12-21 shared-tile index, 22-24/25-27/28-30 tile coordinates
__device__ __forceinline__ uint32_t node_desc(int n) {
    const int t[3] = {n >> 6, (n >> 3) & 7, n & 7};
    uint32_t d = 0;
    int ln = 0, nid = 0;
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        ln = ln * BLK + ((t[a] + 3) & 3);
        nid = nid * 3 + ((t[a] + 3) >> 2);
        d |= (uint32_t)t[a] << (22 + 3 * a);
    }
    d |= (uint32_t)nid << 6;
    d |= (uint32_t)ln;
    d |= (uint32_t)tidx(t[0], t[1], t[2]) << 12;
    return d;
}

// Per-chunk neighbourhood of the chunk's block: global index of block (b + db) and which
// of the 3 offsets per axis are inside the grid.
struct Nbhd {
    int g0;       // global index of the chunk's own block
    int sx, sy;   // block strides (nblk_y * nblk_z, nblk_z)
    uint32_t vx, vy, vz;  // bit (db + 1) set if b + db is inside the grid on that axis
};

__device__ __forceinline__ Nbhd nbhd_of(const mpm_instance& I, const BlockCoord& bc) {
    Nbhd h;
    h.sy = I.nblk[2];
    h.sx = I.nblk[1] * I.nblk[2];
    h.g0 = (int)I.blk_base + bc.bx * h.sx + bc.by * h.sy + bc.bz;
    h.vx = 2u | (bc.bx > 0 ? 1u : 0u) | (bc.bx + 1 < I.nblk[0] ? 4u : 0u);
    h.vy = 2u | (bc.by > 0 ? 1u : 0u) | (bc.by + 1 < I.nblk[1] ? 4u : 0u);
    h.vz = 2u | (bc.bz > 0 ? 1u : 0u) | (bc.bz + 1 < I.nblk[2] ? 4u : 0u);
    return h;
}

// grid address of tile node d, or -1 if its block lies outside the grid
__device__ __forceinline__ int64_t nbhd_addr(const Nbhd& h, uint32_t d) {
    const uint32_t nid = (d >> 6) & 31;
    const uint32_t ex = nid / 9, ey = (nid / 3) % 3, ez = nid % 3;
    if (!((h.vx >> ex) & (h.vy >> ey) & (h.vz >> ez) & 1u)) return -1;
    const int g = h.g0 + ((int)ex - 1) * h.sx + ((int)ey - 1) * h.sy + ((int)ez - 1);
    return ((int64_t)g << 6) + (d & 63);
}

// The 27 neighbour blocks of a work item's block as global block indices (-1 outside the
// grid), by neighbour id, NB_PARTIAL set on blocks that reach past the grid's last node (the
// grid's last block layer, whose padding nodes the flush must not write); threads 0..26
// write one entry each.  With it a tile node's grid address is one shared load and a shift
// from its descriptor.
constexpr int NB_PARTIAL = 1 << 30;

__device__ __forceinline__ void nb_table(const mpm_instance& I, const BlockCoord& bc, int* tab) {
    if (threadIdx.x < 27) {
        const int t = (int)threadIdx.x;
        const int bx = bc.bx + t / 9 - 1, by = bc.by + (t / 3) % 3 - 1, bz = bc.bz + t % 3 - 1;
        const bool in = bx >= 0 && by >= 0 && bz >= 0 && bx < I.nblk[0] && by < I.nblk[1] && bz < I.nblk[2];
        const bool partial = (bx + 1) * BLK > I.res[0] || (by + 1) * BLK > I.res[1] || (bz + 1) * BLK > I.res[2];
        tab[t] = in ? (int)(I.blk_base + (bx * I.nblk[1] + by) * I.nblk[2] + bz) | (partial ? NB_PARTIAL : 0) : -1;
    }
}

__device__ __forceinline__ int64_t tab_addr(const int* tab, uint32_t d) {
    const int blk = tab[(d >> 6) & 31];
    return blk < 0 ? -1 : ((int64_t)(blk & ~NB_PARTIAL) << 6) + (d & 63);
}

// zero the whole tile (once per kernel; the flush re-zeroes what it touched)
__device__ __forceinline__ void tile_zero(Tile& T, int P) {
    for (int n = threadIdx.x; n < TWORDS; n += P) {
        T.t[0][n] = 0;
        T.t[1][n] = 0;
        T.t[2][n] = 0;
        T.t[3][n] = 0;
    }
}

// Chunk-wide fixed-point scales, the marking of the grid blocks the chunk's stencils reach,
// the 27-node scatter and the flush of non-empty nodes to the block-major grid.  Must be
// called by every thread of the CTA (contains barriers); T must be zeroed and a barrier
// passed before.  It ends without a barrier: the flush touches only the tile nodes the
// thread owns (nd), and the next chunk writes the tile only after two more barriers.
template <int P, bool CPIC = false>
__device__ __forceinline__ void scatter_flush(Tile& T, const Payload& o, const mpm_instance& I, int inst,
                                              const BlockCoord& bc, int ox, int oy, int oz, Ws& w, const int* tab,
                                              const uint32_t* nd, const P2GArgs* cp = nullptr) {
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    const float wbq = warp_max(o.in_tile ? o.bq : 0.f);
    const float wbm = warp_max(o.in_tile ? o.mass : 0.f);
    const unsigned nb = __ballot_sync(0xffffffffu, o.in_tile);
    // Reach of the in-tile stencils (base .. base + 2) into the neighbour blocks, per axis:
    // the lower block (tile coordinate 0) iff lx == 0, the upper one (>= 5) iff lx >= 3.
    // Bits 2a / 2a+1: lower / upper neighbour on axis a.
    uint32_t reach = 0u;
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        const int l = o.base[a] - (a == 0 ? ox : (a == 1 ? oy : oz));
        reach |= (__ballot_sync(0xffffffffu, o.in_tile && l == 0) ? 1u : 0u) << (2 * a);
        reach |= (__ballot_sync(0xffffffffu, o.in_tile && l >= 3) ? 2u : 0u) << (2 * a);
    }
    if (lane == 0) {
        T.red[0][wid] = wbq;
        T.red[1][wid] = wbm;
        T.wcnt[wid] = __popc(nb);
        T.wreach[wid] = (int)reach;
    }
    __syncthreads();
    float Bq = 0.f, Bm = 0.f;
    int cnt = 0;
    uint32_t rch = 0u;
#pragma unroll
    for (int i = 0; i < P / 32; ++i) {
        Bq = fmaxf(Bq, T.red[0][i]);
        Bm = fmaxf(Bm, T.red[1][i]);
        cnt += T.wcnt[i];
        rch |= (uint32_t)T.wreach[i];
    }
    // mark the grid blocks the chunk's stencils reach (a superset of the blocks its flush
    // writes: per axis the neighbour is included if any stencil reaches into it)
    if (threadIdx.x < 27 && cnt > 0) {
        const int t = (int)threadIdx.x;
        const int e[3] = {t / 9, (t / 3) % 3, t % 3};  // db + 1 per axis
        bool on = tab[t] >= 0;
#pragma unroll
        for (int a = 0; a < 3; ++a) {
            if (e[a] == 0) on = on && ((rch >> (2 * a)) & 1u);
            if (e[a] == 2) on = on && ((rch >> (2 * a + 1)) & 1u);
        }
        if (on) mark_block(w, inst, I, bc.bx + e[0] - 1, bc.by + e[1] - 1, bc.bz + e[2] - 1);
    }
    const float nin = (float)max(cnt, 256);
    // scale = 2^(29 - floor(log2(n * B))): n * B * scale < 2^30
    const float sq = Bq > 0.f ? ldexpf(1.f, max(-120, min(120, 29 - ilogbf(nin * Bq)))) : 1.f;
    const float sm = Bm > 0.f ? ldexpf(1.f, max(-120, min(120, 29 - ilogbf(nin * Bm)))) : 1.f;
    uint32_t sw[7] = {0u, 0u, 0u, 0u, 0u, 0u, 0u};  // CPIC: separated nodes
    if (o.live) {
        float wx[3], wy[3], wz[3];
        bspline(o.fx[0], wx);
        bspline(o.fx[1], wy);
        bspline(o.fx[2], wz);
        if (o.in_tile) {
            const int lx = o.base[0] - ox, ly = o.base[1] - oy, lz = o.base[2] - oz;
            const float mq0 = o.q[0] * sq, mq1 = o.q[1] * sq, mq2 = o.q[2] * sq, ms = o.mass * sm;
            float As[9];
#pragma unroll
            for (int k = 0; k < 9; ++k) As[k] = o.A[k] * sq;
            if constexpr (kF32x2Scatter<P> && !CPIC) {
                // the same arithmetic on lane pairs: (momentum x, momentum y) and (momentum z,
                // mass); the mass lane's affine coefficients are 0, so it stays ms exactly
                constexpr float kMagic = 12582912.0f;  // 1.5 * 2^23: round-to-nearest integer
                const float2 q01 = make_float2(mq0, mq1), q2m = make_float2(mq2, ms);
                const float2 Ax = make_float2(As[0], As[3]), Ax2 = make_float2(As[6], 0.f);
                const float2 Ay = make_float2(As[1], As[4]), Ay2 = make_float2(As[7], 0.f);
                const float2 Az = make_float2(As[2], As[5]), Az2 = make_float2(As[8], 0.f);
#pragma unroll kOuterUnroll
                for (int i = 0; i < 3; ++i) {
                    const float2 fi = dup2((float)i), wxi = dup2(sel3(wx, i));
                    const float2 b01 = fma2(Ax, fi, q01), b2m = fma2(Ax2, fi, q2m);
#pragma unroll
                    for (int j = 0; j < 3; ++j) {
                        const float2 fj = dup2((float)j);
                        const float2 wij = __fmul2_rn(wxi, dup2(wy[j]));
                        const float2 c01 = fma2(Ay, fj, b01), c2m = fma2(Ay2, fj, b2m);
                        const int row = tidx(lx + i, ly + j, lz);
#pragma unroll
                        for (int k = 0; k < 3; ++k) {
                            const float2 fk = dup2((float)k);
                            const float2 wt = __fmul2_rn(wij, dup2(wz[k]));
                            const float2 r01 = fma2(wt, fma2(Az, fk, c01), dup2(kMagic));
                            const float2 r2m = fma2(wt, fma2(Az2, fk, c2m), dup2(kMagic));
                            atomicAdd(&T.t[0][row + k], __float_as_int(r01.x) - 0x4B400000);
                            atomicAdd(&T.t[1][row + k], __float_as_int(r01.y) - 0x4B400000);
                            atomicAdd(&T.t[2][row + k], __float_as_int(r2m.x) - 0x4B400000);
                            atomicAdd(&T.t[3][row + k], __float_as_int(r2m.y) - 0x4B400000);
                        }
                    }
                }
            } else {
            // factored per axis: the (i, j) partial sums and weights are reused for the 3 k
#pragma unroll kOuterUnroll
            for (int i = 0; i < 3; ++i) {
                const float wxi = sel3(wx, i), fi = (float)i;
                const float b0 = mq0 + As[0] * fi, b1 = mq1 + As[3] * fi, b2 = mq2 + As[6] * fi;
#pragma unroll
                for (int j = 0; j < 3; ++j) {
                    const float wij = wxi * wy[j];
                    const float c0 = b0 + As[1] * j, c1 = b1 + As[4] * j, c2 = b2 + As[7] * j;
                    const int row = tidx(lx + i, ly + j, lz);
#pragma unroll
                    for (int k = 0; k < 3; ++k) {
                        const float wt = wij * wz[k];
                        if constexpr (CPIC) {
                            const uint32_t sg =
                                cpic_separating(*cp, inst, I, o.gid, o.base[0] + i, o.base[1] + j, o.base[2] + k);
                            if (sg) {
                                const int nidx = i * 9 + j * 3 + k;
                                sw[nidx >> 2] |= sg << (8 * (nidx & 3));
                                continue;
                            }
                        }
                        atomicAdd(&T.t[0][row + k], fix_mul(wt, c0 + As[2] * k));
                        atomicAdd(&T.t[1][row + k], fix_mul(wt, c1 + As[5] * k));
                        atomicAdd(&T.t[2][row + k], fix_mul(wt, c2 + As[8] * k));
                        atomicAdd(&T.t[3][row + k], fix_mul(wt, ms));
                    }
                }
            }
            }
        } else {
            // drifted since the last sort (or a non-finite stress): bounds-checked global path
            atomicAdd((unsigned long long*)&w.counters[CNT_FALLBACK], 1ull);
#pragma unroll 1
            for (int i = 0; i < 3; ++i)
#pragma unroll 1
                for (int j = 0; j < 3; ++j)
#pragma unroll 1
                    for (int k = 0; k < 3; ++k) {
                        const int gx = o.base[0] + i, gy = o.base[1] + j, gz = o.base[2] + k;
                        if (gx < 0 || gy < 0 || gz < 0 || gx >= I.res[0] || gy >= I.res[1] || gz >= I.res[2]) {
                            set_status(w, inst, MPM_STATUS_OUT_OF_GRID);
                            continue;
                        }
                        if constexpr (CPIC) {
                            const uint32_t sg = cpic_separating(*cp, inst, I, o.gid, gx, gy, gz);
                            if (sg) {
                                const int nidx = i * 9 + j * 3 + k;
                                sw[nidx >> 2] |= sg << (8 * (nidx & 3));
                                continue;
                            }
                        }
                        const float wt = sel3(wx, i) * sel3(wy, j) * sel3(wz, k);
                        const float ax = o.q[0] + (o.A[0] * i + o.A[1] * j + o.A[2] * k);
                        const float ay = o.q[1] + (o.A[3] * i + o.A[4] * j + o.A[5] * k);
                        const float az = o.q[2] + (o.A[6] * i + o.A[7] * j + o.A[8] * k);
                        atomicAdd(&w.mm[node_addr(I, gx, gy, gz)], make_float4(wt * ax, wt * ay, wt * az, wt * o.mass));
                        mark_block(w, inst, I, gx >> 2, gy >> 2, gz >> 2);
                    }
        }
    }
    if constexpr (CPIC) {
        if (o.slot >= 0) cpic_store(*cp, o.slot, sw);
    }
    __syncthreads();
    // flush non-empty tile nodes, one 16-byte reduction each, zeroing the tile behind it
    const float iq = 1.f / sq, im = 1.f / sm;
#pragma unroll
    for (int k = 0; k < TN / P; ++k) {
        const uint32_t d = nd[threadIdx.x + k * P];
        const int t = (d >> 12) & 1023;
        const int mi = T.t[3][t], m0 = T.t[0][t], m1 = T.t[1][t], m2 = T.t[2][t];
        if ((mi | m0 | m1 | m2) != 0) {
            const int e = tab[(d >> 6) & 31];
            bool ok = e >= 0;
            if (ok && (e & NB_PARTIAL)) {
                // a block of the grid's last layer: its padding nodes lie outside the grid
                const int tx = (d >> 22) & 7, ty = (d >> 25) & 7, tz = (d >> 28) & 7;
                ok = ox + tx < I.res[0] && oy + ty < I.res[1] && oz + tz < I.res[2];
            }
            if (!ok) {
                set_status(w, inst, MPM_STATUS_OUT_OF_GRID);
            } else {
                const int64_t a = ((int64_t)(e & ~NB_PARTIAL) << 6) + (d & 63);
                atomicAdd(&w.mm[a], make_float4((float)m0 * iq, (float)m1 * iq, (float)m2 * iq, (float)mi * im));
            }
            T.t[0][t] = 0;
            T.t[1][t] = 0;
            T.t[2][t] = 0;
            T.t[3][t] = 0;
        }
    }
}

template <int P>
__device__ __forceinline__ void vel_tile_load_tab(VelTile& VT, const Ws& w, const int* tab, const uint32_t* nd) {
#pragma unroll
    for (int k = 0; k < TN / P; ++k) {
        const uint32_t d = nd[threadIdx.x + k * P];
        const int64_t a = tab_addr(tab, d);
        // the velocity tile has the scatter tile's layout, so the descriptor's tile index serves
        VT.v[(d >> 12) & 1023] = a >= 0 ? w.gv[a] : make_float4(0.f, 0.f, 0.f, 0.f);
    }
}

template <int P>
__device__ __forceinline__ void vel_tile_load(VelTile& VT, const Ws& w, const Nbhd& h, const uint32_t* nd) {
#pragma unroll
    for (int k = 0; k < TN / P; ++k) {
        const uint32_t d = nd[threadIdx.x + k * P];
        const int64_t a = nbhd_addr(h, d);
        VT.v[vidx((d >> 22) & 7, (d >> 25) & 7, (d >> 28) & 7)] = a >= 0 ? w.gv[a] : make_float4(0.f, 0.f, 0.f, 0.f);
    }
}

// g2p gather (mpm_solver.py:396-431): v = sum w v_i, C = 4 inv_dx sum w v_i (off - fx)^T;
// then x += dt v and the boundary (mpm_solver.py:434-437).  Returns false if nothing
// could be gathered (non-finite x).
template <int P, bool CPIC = false>
__device__ __forceinline__ bool gather(const VelTile& VT, const Ws& w, const mpm_instance& I, int inst, float* x,
                                       float* nv, float* nC, int ox, int oy, int oz, const P2GArgs* cp = nullptr,
                                       int p = 0) {
    if (!finite3(x[0], x[1], x[2])) {
        set_status(w, inst, MPM_STATUS_NAN);
        return false;
    }
    float fx[3], wx[3], wy[3], wz[3];
    int base[3];
    locate(I, x, base, fx);
    bspline(fx[0], wx);
    bspline(fx[1], wy);
    bspline(fx[2], wz);
    nv[0] = nv[1] = nv[2] = 0.f;
#pragma unroll
    for (int k = 0; k < 9; ++k) nC[k] = 0.f;
    if (tile_contains(base, ox, oy, oz)) {
        // separable evaluation: reduce along z, then y, then x.  With u = off - fx,
        // C_ab = c sum_ijk w v_a u_b factors per axis, so each node costs one load and six
        // FMAs instead of twelve.
        const int lx = base[0] - ox, ly = base[1] - oy, lz = base[2] - oz;
        float wzd[3], wyd[3], wxd[3];
#pragma unroll
        for (int k = 0; k < 3; ++k) {
            wzd[k] = wz[k] * ((float)k - fx[2]);
            wyd[k] = wy[k] * ((float)k - fx[1]);
            wxd[k] = wx[k] * ((float)k - fx[0]);
        }
        if constexpr (kF32x2Gather<P>) {
            // the same sums on lane pairs: (x, y) of every sum, and for z the pairs (s0, s1),
            // (a0, az), (vp, c2), whose two lanes take the same node value: the tile's w holds
            // a copy of z (k_grid_op stores (vx, vy, vz, vz)), so (g.z, g.w) is that pair as loaded
            const float2 z2 = make_float2(0.f, 0.f);
            float2 vp = z2, c0 = z2, c1 = z2, c2 = z2, vc2z = z2;
            float c0z = 0.f, c1z = 0.f;
            const float2 wzp[3] = {make_float2(wz[0], wzd[0]), make_float2(wz[1], wzd[1]), make_float2(wz[2], wzd[2])};
#pragma unroll kOuterUnroll
            for (int i = 0; i < 3; ++i) {
                float2 a0 = z2, ay = z2, az = z2, a0azz = z2;
                float ayz = 0.f;
#pragma unroll
                for (int j = 0; j < 3; ++j) {
                    float2 s0 = z2, s1 = z2, s01z = z2;
#pragma unroll
                    for (int k = 0; k < 3; ++k) {
                        const float4 g = VT.v[vidx(lx + i, ly + j, lz + k)];
                        const float2 gxy = make_float2(g.x, g.y);
                        s0 = fma2(dup2(wz[k]), gxy, s0);
                        s1 = fma2(dup2(wzd[k]), gxy, s1);
                        s01z = fma2(wzp[k], make_float2(g.z, g.w), s01z);
                    }
                    const float2 wj = dup2(wy[j]), wdj = dup2(wyd[j]);
                    a0 = fma2(wj, s0, a0);
                    ay = fma2(wdj, s0, ay);
                    az = fma2(wj, s1, az);
                    a0azz = fma2(wj, s01z, a0azz);
                    ayz = fmaf(wyd[j], s01z.x, ayz);
                }
                const float2 wi = dup2(sel3(wx, i)), wdi = dup2(sel3(wxd, i));
                vp = fma2(wi, a0, vp);
                c0 = fma2(wdi, a0, c0);
                c1 = fma2(wi, ay, c1);
                c2 = fma2(wi, az, c2);
                vc2z = fma2(wi, a0azz, vc2z);
                c0z = fmaf(sel3(wxd, i), a0azz.x, c0z);
                c1z = fmaf(sel3(wx, i), ayz, c1z);
            }
            nv[0] = vp.x;
            nv[1] = vp.y;
            nv[2] = vc2z.x;
            const float2 cs = dup2(I.c_scale);
            c0 = __fmul2_rn(c0, cs);
            c1 = __fmul2_rn(c1, cs);
            c2 = __fmul2_rn(c2, cs);
            nC[0] = c0.x;
            nC[1] = c1.x;
            nC[2] = c2.x;
            nC[3] = c0.y;
            nC[4] = c1.y;
            nC[5] = c2.y;
            nC[6] = c0z * I.c_scale;
            nC[7] = c1z * I.c_scale;
            nC[8] = vc2z.y * I.c_scale;
        } else {
#pragma unroll kOuterUnroll
        for (int i = 0; i < 3; ++i) {
            float a0[3] = {0.f, 0.f, 0.f}, ay[3] = {0.f, 0.f, 0.f}, az[3] = {0.f, 0.f, 0.f};
#pragma unroll
            for (int j = 0; j < 3; ++j) {
                float s0[3] = {0.f, 0.f, 0.f}, s1[3] = {0.f, 0.f, 0.f};
#pragma unroll
                for (int k = 0; k < 3; ++k) {
                    const float4 g = VT.v[vidx(lx + i, ly + j, lz + k)];
                    s0[0] += wz[k] * g.x;
                    s0[1] += wz[k] * g.y;
                    s0[2] += wz[k] * g.z;
                    s1[0] += wzd[k] * g.x;
                    s1[1] += wzd[k] * g.y;
                    s1[2] += wzd[k] * g.z;
                }
#pragma unroll
                for (int a = 0; a < 3; ++a) {
                    a0[a] += wy[j] * s0[a];
                    ay[a] += wyd[j] * s0[a];
                    az[a] += wy[j] * s1[a];
                }
            }
            const float wxi = sel3(wx, i), wxdi = sel3(wxd, i);
#pragma unroll
            for (int a = 0; a < 3; ++a) {
                nv[a] += wxi * a0[a];
                nC[a * 3 + 0] += wxdi * a0[a];
                nC[a * 3 + 1] += wxi * ay[a];
                nC[a * 3 + 2] += wxi * az[a];
            }
        }
#pragma unroll
        for (int k = 0; k < 9; ++k) nC[k] *= I.c_scale;
        }
    } else {
#pragma unroll 1
        for (int i = 0; i < 3; ++i)
#pragma unroll 1
            for (int j = 0; j < 3; ++j)
#pragma unroll 1
                for (int k = 0; k < 3; ++k) {
                    const int gx = base[0] + i, gy = base[1] + j, gz = base[2] + k;
                    if (gx < 0 || gy < 0 || gz < 0 || gx >= I.res[0] || gy >= I.res[1] || gz >= I.res[2]) {
                        set_status(w, inst, MPM_STATUS_OUT_OF_GRID);
                        continue;
                    }
                    const float4 g = w.gv[node_addr(I, gx, gy, gz)];
                    const float wt = sel3(wx, i) * sel3(wy, j) * sel3(wz, k);
                    const float d0 = (float)i - fx[0], d1 = (float)j - fx[1], d2 = (float)k - fx[2];
                    nv[0] += wt * g.x;
                    nv[1] += wt * g.y;
                    nv[2] += wt * g.z;
                    const float cw = I.c_scale * wt;
                    nC[0] += cw * g.x * d0;
                    nC[1] += cw * g.x * d1;
                    nC[2] += cw * g.x * d2;
                    nC[3] += cw * g.y * d0;
                    nC[4] += cw * g.y * d1;
                    nC[5] += cw * g.y * d2;
                    nC[6] += cw * g.z * d0;
                    nC[7] += cw * g.z * d1;
                    nC[8] += cw * g.z * d2;
                }
    }
    if constexpr (CPIC)
        cpic_correct(*cp, &VT, w, I, p, x, base, fx, wx, wy, wz, tile_contains(base, ox, oy, oz), ox, oy, oz, nv, nC);
    // a non-finite velocity is flagged separately: the boundary clamp (fminf/fmaxf, like
    // ti.min/ti.max) maps a NaN position back onto the wall, so the reference's
    // position-only check would not see it
    if (!finite3(nv[0], nv[1], nv[2])) set_status(w, inst, MPM_STATUS_NONFINITE_VEL);
#pragma unroll
    for (int d = 0; d < 3; ++d) {
        const float nx = x[d] + I.dt * nv[d];
        nv[d] = bc_vel(nx, nv[d], I.bnd_lo[d], I.bnd_hi[d]);
        x[d] = fmaxf(fminf(nx, I.bnd_hi[d]), I.bnd_lo[d]);
    }
    if (!finite3(x[0], x[1], x[2])) set_status(w, inst, MPM_STATUS_NAN);
    return true;
}

// ---------------------------------------------------------------- p2g

template <int P, bool MUSCLE, bool CPIC>
__global__ void __launch_bounds__(P, kP2GCtasPerSM<P>) k_p2g(P2GArgs a) {
    __shared__ Tile T;
    __shared__ Stash<P> SH;
    Ws& w = a.w;
    const int n_chunks = (int)w.counters[CNT_CHUNKS];
    const int64_t st = a.par.state_stride;
    const float* __restrict__ S = a.par.state;
    __shared__ uint32_t nd[TN];  // each thread reads back only the entries it wrote
#pragma unroll
    for (int k = 0; k < TN / P; ++k) nd[threadIdx.x + k * P] = node_desc(threadIdx.x + k * P);
    tile_zero(T, P);
    // the item's neighbour-block table, first read behind the scatter's first barrier; two
    // buffers, as the previous item's flush may still read its own
    __shared__ int nbt[2][27];
    int tb = 0;
    for (int ci = blockIdx.x; ci < n_chunks; ci += gridDim.x) {
        const int4 ch = w.chunks[ci];
        const mpm_instance& I = a.inst[ch.x];
        const BlockCoord bc = unpack_bc(ch.y);
        nb_table(I, bc, nbt[tb]);
        const int ox = bc.bx * BLK - MARGIN, oy = bc.by * BLK - MARGIN, oz = bc.bz * BLK - MARGIN;
        Payload o;
        o.live = o.in_tile = false;
        o.mass = o.bq = 0.f;
        o.slot = -1;
        const int p = ch.z + threadIdx.x;
        if (p < ch.w && (a.par.pflags[p] & MPM_PFLAG_ACTIVE)) {
            float x[3], v[3], C[9];
#pragma unroll
            for (int d = 0; d < 3; ++d) {
                x[d] = __ldg(&S[(MPM_CH_X + d) * st + p]);
                v[d] = __ldg(&S[(MPM_CH_V + d) * st + p]);
            }
#pragma unroll
            for (int k = 0; k < 9; ++k) C[k] = __ldg(&S[(MPM_CH_C + k) * st + p]);
            if constexpr (CPIC) {
                o.slot = p;
                o.gid = a.par.gid[p];
                cpic_update_normals(a, ch.x, I, o.gid, x);
            }
            particle_update<P, MUSCLE>(I, a.mats, a.par, p, x, v, C, ox, oy, oz, o, w, ch.x, SH);
        }
        scatter_flush<P, CPIC>(T, o, I, ch.x, bc, ox, oy, oz, w, nbt[tb], nd, &a);
        tb ^= 1;
    }
}

// ---------------------------------------------------------------- g2p

template <int P, bool CPIC>
__global__ void __launch_bounds__(P, 1024 / P) k_g2p(P2GArgs a) {
    __shared__ VelTile VT;
    Ws& w = a.w;
    const int n_chunks = (int)w.counters[CNT_CHUNKS];
    const int64_t st = a.par.state_stride;
    float* __restrict__ S = a.par.state;
    __shared__ uint32_t nd[TN];  // each thread reads back only the entries it wrote
#pragma unroll
    for (int k = 0; k < TN / P; ++k) nd[threadIdx.x + k * P] = node_desc(threadIdx.x + k * P);
    for (int ci = blockIdx.x; ci < n_chunks; ci += gridDim.x) {
        const int4 ch = w.chunks[ci];
        const mpm_instance& I = a.inst[ch.x];
        const BlockCoord bc = unpack_bc(ch.y);
        const Nbhd h = nbhd_of(I, bc);
        const int ox = bc.bx * BLK - MARGIN, oy = bc.by * BLK - MARGIN, oz = bc.bz * BLK - MARGIN;
        vel_tile_load<P>(VT, w, h, nd);
        __syncthreads();
        const int p = ch.z + threadIdx.x;
        if (p < ch.w && (a.par.pflags[p] & MPM_PFLAG_ACTIVE)) {
            float x[3], nv[3], nC[9];
#pragma unroll
            for (int d = 0; d < 3; ++d) x[d] = S[(MPM_CH_X + d) * st + p];
            if (gather<P, CPIC>(VT, w, I, ch.x, x, nv, nC, ox, oy, oz, &a, p)) {
#pragma unroll
                for (int d = 0; d < 3; ++d) {
                    S[(MPM_CH_X + d) * st + p] = x[d];
                    S[(MPM_CH_V + d) * st + p] = nv[d];
                }
#pragma unroll
                for (int k = 0; k < 9; ++k) S[(MPM_CH_C + k) * st + p] = nC[k];
            }
        }
        __syncthreads();
    }
}

// ---------------------------------------------------------------- fused g2p + p2g

// g2p of substep n fused with p2g of substep n+1: the new v and C never leave registers
// (they are recomputed from the grid by the next gather), only x, F and Jp are stored.
template <int P, bool MUSCLE, bool CPIC>
__global__ void __launch_bounds__(P, kP2GCtasPerSM<P>) k_g2p2g(P2GArgs a) {
    __shared__ VelTile VT;
    __shared__ Tile T;
    __shared__ Stash<P> SH;
    Ws& w = a.w;
    const int n_chunks = (int)w.counters[CNT_CHUNKS];
    const int64_t st = a.par.state_stride;
    float* __restrict__ S = a.par.state;
    __shared__ uint32_t nd[TN];  // each thread reads back only the entries it wrote
#pragma unroll
    for (int k = 0; k < TN / P; ++k) nd[threadIdx.x + k * P] = node_desc(threadIdx.x + k * P);
    tile_zero(T, P);
    // the next work item's descriptor is loaded one item ahead, and each item's particle
    // position and flags are in flight during its velocity-tile load: the item start's chain of
    // dependent loads (descriptor -> tile; then position -> gather) loses two L2 round trips
    int4 next = blockIdx.x < n_chunks ? w.chunks[blockIdx.x] : make_int4(0, 0, 0, 0);
    // neighbour-block tables (global block index per neighbour id): each item's is built during
    // the item before (behind that item's tile barrier; read at this item's tile load and flush)
    __shared__ int nbt[2][27];
    int tb = 0;
    if ((int)blockIdx.x < n_chunks) nb_table(a.inst[next.x], unpack_bc(next.y), nbt[0]);
    __syncthreads();
    for (int ci = blockIdx.x; ci < n_chunks; ci += gridDim.x) {
        const int4 ch = next;
        if (ci + (int)gridDim.x < n_chunks) next = w.chunks[ci + gridDim.x];
        const int p = ch.z + threadIdx.x;
        const bool have = p < ch.w;
        float x[3] = {0.f, 0.f, 0.f};
        uint8_t pf = 0;
        if (have) {
            pf = a.par.pflags[p];
#pragma unroll
            for (int d = 0; d < 3; ++d) x[d] = S[(MPM_CH_X + d) * st + p];
        }
        const mpm_instance& I = a.inst[ch.x];
        const BlockCoord bc = unpack_bc(ch.y);
        const int ox = bc.bx * BLK - MARGIN, oy = bc.by * BLK - MARGIN, oz = bc.bz * BLK - MARGIN;
        vel_tile_load_tab<P>(VT, w, nbt[tb], nd);
        __syncthreads();
        // the other table was last read by the previous item's flush, before this barrier
        if (ci + (int)gridDim.x < n_chunks) nb_table(a.inst[next.x], unpack_bc(next.y), nbt[tb ^ 1]);
        Payload o;
        o.live = o.in_tile = false;
        o.mass = o.bq = 0.f;
        o.slot = -1;
        if (have && (pf & MPM_PFLAG_ACTIVE)) {
            float nv[3], nC[9];
            if constexpr (CPIC) o.slot = p;  // a particle with a non-finite x leaves no separated nodes
            if (gather<P, CPIC>(VT, w, I, ch.x, x, nv, nC, ox, oy, oz, &a, p)) {
#pragma unroll
                for (int d = 0; d < 3; ++d) S[(MPM_CH_X + d) * st + p] = x[d];
                if constexpr (CPIC) {
                    // the next g2p's rigid response needs this substep's velocity, and the
                    // normals follow the particle after its gather (coupler.preprocess)
#pragma unroll
                    for (int d = 0; d < 3; ++d) S[(MPM_CH_V + d) * st + p] = nv[d];
                    o.gid = a.par.gid[p];
                    cpic_update_normals(a, ch.x, I, o.gid, x);
                }
                particle_update<P, MUSCLE>(I, a.mats, a.par, p, x, nv, nC, ox, oy, oz, o, w, ch.x, SH);
            }
        }
        scatter_flush<P, CPIC>(T, o, I, ch.x, bc, ox, oy, oz, w, nbt[tb], nd, &a);
        tb ^= 1;
    }
}

// non-free particles zero the momentum of their stencil (mpm_solver.py:388-389)
__global__ void k_nonfree_zero(mpm_problem prob, const mpm_instance* __restrict__ inst, mpm_particles par, Ws w) {
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= prob.n_particles) return;
    const uint8_t fl = par.pflags[p];
    if (!(fl & MPM_PFLAG_ACTIVE) || (fl & MPM_PFLAG_FREE)) return;
    const int k = find_instance_by_particle(inst, prob.n_instances, p);
    const mpm_instance& I = inst[k];
    const int64_t st = par.state_stride;
    int base[3];
    for (int d = 0; d < 3; ++d) {
        const float x = par.state[(MPM_CH_X + d) * st + p];
        if (!isfinite(x)) return;
        base[d] = (int)fminf(fmaxf(floorf(x * I.inv_dx - 0.5f), -1e8f), 1e8f) - I.lower_cell[d];
    }
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j)
            for (int kk = 0; kk < 3; ++kk) {
                const int gx = base[0] + i, gy = base[1] + j, gz = base[2] + kk;
                if (gx < 0 || gy < 0 || gz < 0 || gx >= I.res[0] || gy >= I.res[1] || gz >= I.res[2]) continue;
                float4* c = &w.mm[node_addr(I, gx, gy, gz)];
                c->x = 0.f;
                c->y = 0.f;
                c->z = 0.f;
            }
}

// ---------------------------------------------------------------- grid op

// constant-velocity kinematic motion of the colliders over one substep of their instance:
// pos += lin_vel dt (a tool's origin then clamped to its floor, tool_entity.py:178-189),
// rot = exp([ang_vel] dt) rot
__global__ void k_advance_colliders(const mpm_instance* __restrict__ inst, int n_inst, mpm_collider* cs, int n) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    mpm_collider& c = cs[i];
    if (c.instance < 0 || c.instance >= n_inst) return;
    const float dt = inst[c.instance].dt;
#pragma unroll
    for (int d = 0; d < 3; ++d) c.pos[d] += c.lin_vel[d] * dt;
    if (c.kind == MPM_COLLIDER_TOOL) c.pos[2] = fmaxf(c.pos[2], c.floor);
    if (c.ang_vel[0] != 0.f || c.ang_vel[1] != 0.f || c.ang_vel[2] != 0.f) {
        float E[9], R[9];
        rot_step(c.ang_vel, dt, E);
#pragma unroll
        for (int a = 0; a < 3; ++a)
#pragma unroll
            for (int b = 0; b < 3; ++b)
                R[a * 3 + b] = E[a * 3 + 0] * c.rot[0 * 3 + b] + E[a * 3 + 1] * c.rot[1 * 3 + b] + E[a * 3 + 2] * c.rot[2 * 3 + b];
#pragma unroll
        for (int k = 0; k < 9; ++k) c.rot[k] = R[k];
    }
}

// ---------------------------------------------------------------- force fields
// engine/force_fields.py, applied by the grid op (legacy_coupler.py:377-379)

// splitmix64's output function (Steele, Lea and Flood, OOPSLA 2014): a well-mixed 64-bit
// value per 64-bit key, the counter-based uniform source of the NOISE field
__device__ __forceinline__ uint64_t mix64(uint64_t z) {
    z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ull;
    z = (z ^ (z >> 27)) * 0x94d049bb133111ebull;
    return z ^ (z >> 31);
}

// Ken Perlin's improved noise (2002), as PerlinNoiseField._noise (force_fields.py:441-540)
// states it over a 512-entry permutation table P (a 256-permutation written twice)
__device__ __forceinline__ float perlin_fade(float t) { return t * t * t * (t * (t * 6.f - 15.f) + 10.f); }
__device__ __forceinline__ float perlin_lerp(float t, float a, float b) { return a + t * (b - a); }
__device__ __forceinline__ float perlin_grad(int h, float x, float y, float z) {
    h &= 15;
    const float u = h < 8 ? x : y;
    const float v = h < 4 ? y : ((h == 12 || h == 14) ? x : z);
    return ((h & 1) ? -u : u) + ((h & 2) ? -v : v);
}
__device__ float perlin(const int* __restrict__ P, float freq, float x, float y, float z) {
    x *= freq;
    y *= freq;
    z *= freq;
    const float fx = floorf(x), fy = floorf(y), fz = floorf(z);
    const int X = (int)fx & 255, Y = (int)fy & 255, Z = (int)fz & 255;
    x -= fx;
    y -= fy;
    z -= fz;
    const float u = perlin_fade(x), v = perlin_fade(y), w = perlin_fade(z);
    const int A = P[X] + Y, AA = P[A] + Z, AB = P[A + 1] + Z;
    const int B = P[X + 1] + Y, BA = P[B] + Z, BB = P[B + 1] + Z;
    return perlin_lerp(
        w,
        perlin_lerp(v, perlin_lerp(u, perlin_grad(P[AA], x, y, z), perlin_grad(P[BA], x - 1.f, y, z)),
                    perlin_lerp(u, perlin_grad(P[AB], x, y - 1.f, z), perlin_grad(P[BB], x - 1.f, y - 1.f, z))),
        perlin_lerp(v,
                    perlin_lerp(u, perlin_grad(P[AA + 1], x, y, z - 1.f), perlin_grad(P[BA + 1], x - 1.f, y, z - 1.f)),
                    perlin_lerp(u, perlin_grad(P[AB + 1], x, y - 1.f, z - 1.f),
                                perlin_grad(P[BB + 1], x - 1.f, y - 1.f, z - 1.f))));
}

// POINT's falloff 1 / (sqrt(|r|^2 + eps) + 1)^falloff_pow and VORTEX's, shared by the adjoint
__device__ __forceinline__ float point_falloff(const mpm_force_field& f, float eps, const float* p) {
    const float r[3] = {p[0] - f.vec[0], p[1] - f.vec[1], p[2] - f.vec[2]};
    return 1.f / powf(sqrtf(r[0] * r[0] + r[1] * r[1] + r[2] * r[2] + eps) + 1.f, f.falloff_pow);
}
__device__ __forceinline__ float vortex_falloff(const mpm_force_field& f, float rho) {
    if (rho < f.falloff_min) return 1.f;
    if (rho < f.falloff_max) return 1.f / powf(rho - f.falloff_min + 1.f, f.falloff_pow);
    return 0.f;
}

// acceleration of one (active) field at node p with velocity v; node / ops key the NOISE draw
__device__ void force_field_acc(const mpm_force_field& f, const int* __restrict__ perm, float eps, const float* p,
                                const float* v, int64_t node, uint32_t ops, float* acc) {
    acc[0] = acc[1] = acc[2] = 0.f;
    switch (f.kind) {
        case MPM_FF_CONSTANT:
            acc[0] = f.vec[0];
            acc[1] = f.vec[1];
            acc[2] = f.vec[2];
            break;
        case MPM_FF_WIND: {
            const float q[3] = {p[0] - f.center[0], p[1] - f.center[1], p[2] - f.center[2]};
            const float c[3] = {q[1] * f.dir[2] - q[2] * f.dir[1], q[2] * f.dir[0] - q[0] * f.dir[2],
                                q[0] * f.dir[1] - q[1] * f.dir[0]};
            if (!(sqrtf(c[0] * c[0] + c[1] * c[1] + c[2] * c[2]) > f.radius)) {
                acc[0] = f.vec[0];
                acc[1] = f.vec[1];
                acc[2] = f.vec[2];
            }
            break;
        }
        case MPM_FF_POINT: {
            const float r[3] = {p[0] - f.vec[0], p[1] - f.vec[1], p[2] - f.vec[2]};
            const float rad = sqrtf(r[0] * r[0] + r[1] * r[1] + r[2] * r[2] + eps);
            const float fo = 1.f / powf(rad + 1.f, f.falloff_pow);
#pragma unroll
            for (int d = 0; d < 3; ++d) {
                const float a = f.strength * r[d] / rad;
                acc[d] = (a + (a - v[d]) * f.flow) * fo;
            }
            break;
        }
        case MPM_FF_DRAG: {
            const float vn = sqrtf(v[0] * v[0] + v[1] * v[1] + v[2] * v[2]);
#pragma unroll
            for (int d = 0; d < 3; ++d) acc[d] = -f.linear * v[d] - f.quadratic * vn * v[d];
            break;
        }
        case MPM_FF_NOISE: {
            const uint64_t h = mix64(mix64(((uint64_t)f.seed << 32) | ops) ^ (uint64_t)node);
#pragma unroll
            for (int d = 0; d < 3; ++d) {
                const float u = (float)(mix64(h + (uint64_t)d) >> 40) * (1.f / 16777216.f);
                acc[d] = (u * 2.f - 1.f) * f.strength;
            }
            break;
        }
        case MPM_FF_VORTEX: {
            const float rx = p[0] - f.center[0], ry = p[1] - f.center[1];
            const float fo = vortex_falloff(f, sqrtf(rx * rx + ry * ry));
            acc[0] = fo * (f.strength * -ry + f.strength2 * -rx) - f.damping * v[0];
            acc[1] = fo * (f.strength * rx + f.strength2 * -ry) - f.damping * v[1];
            acc[2] = -f.damping * v[2];
            break;
        }
        case MPM_FF_TURBULENCE: {
            if (!perm) break;
            const int* P = perm + f.perm_offset;
#pragma unroll
            for (int d = 0; d < 3; ++d) {
                const float a = perlin(P + 512 * d, f.frequency, p[0], p[1], p[2]) * f.strength;
                acc[d] = a + (a - v[d]) * f.flow;
            }
            break;
        }
        default:
            break;
    }
}

// v += acc dt for every active field in order (each sees the velocity the previous ones left)
__device__ __forceinline__ void apply_force_fields(const mpm_force_field* __restrict__ ffs, int n, const int* perm,
                                                   float eps, float dt, const float* p, float* v, int64_t node,
                                                   uint32_t ops) {
    for (int k = 0; k < n; ++k) {
        if (!ffs[k].active) continue;
        float a[3];
        force_field_acc(ffs[k], perm, eps, p, v, node, ops, a);
        v[0] += a[0] * dt;
        v[1] += a[1] * dt;
        v[2] += a[2] * dt;
    }
}

// at most 64 registers (4 CTAs per SM): the collider responses, rare, may spill instead.
// FF: the problem has force fields (a separate instantiation keeps their registers out of
// the common path)
template <bool FF>
__global__ void __launch_bounds__(256, 4) k_grid_op(mpm_problem prob, const mpm_instance* __restrict__ inst, Ws w,
                                                 const mpm_collider* __restrict__ colliders, int n_colliders,
                                                 float* collider_force, const float* __restrict__ sdf_voxels,
                                                 const mpm_force_field* __restrict__ ffs, int n_ff,
                                                 const int* __restrict__ ff_perm, int count_op) {
    const int n_active = (int)w.counters[CNT_ACTIVE];
    const uint32_t ops = w.counters[CNT_GRID_OPS];
    const int gpc = blockDim.x / BLK3;
    const int grp = threadIdx.x / BLK3;
    const int ln = threadIdx.x % BLK3;
    const int lx = ln / (BLK * BLK), ly = (ln / BLK) % BLK, lz = ln % BLK;
    for (int i = blockIdx.x * gpc + grp; i < n_active; i += gridDim.x * gpc) {
        const int2 e = w.active[i];
        const mpm_instance& I = inst[e.x];
        const BlockCoord bc = unpack_bc(e.y);
        const int lb = local_block(I, bc.bx, bc.by, bc.bz);
        const int64_t g = (I.blk_base + lb) * BLK3 + ln;
        const float4 mm = w.mm[g];
        float vx = 0.f, vy = 0.f, vz = 0.f;
        if (mm.w > I.eps) {
            const float inv = 1.f / mm.w;  // (1 / mass) * vel_in (legacy_coupler.py:369)
            vx = inv * mm.x + I.dt * I.gravity[0];
            vy = inv * mm.y + I.dt * I.gravity[1];
            vz = inv * mm.z + I.dt * I.gravity[2];
            // pos = (I + grid_offset) * dx (legacy_coupler.py:374)
            const float px = (float)(bc.bx * BLK + lx + I.lower_cell[0]) * I.dx;
            const float py = (float)(bc.by * BLK + ly + I.lower_cell[1]) * I.dx;
            const float pz = (float)(bc.bz * BLK + lz + I.lower_cell[2]) * I.dx;
            if (FF && n_ff > 0) {  // external force fields (legacy_coupler.py:377-379)
                const float p[3] = {px, py, pz};
                float v[3] = {vx, vy, vz};
                apply_force_fields(ffs, n_ff, ff_perm, I.eps, I.dt, p, v, g, ops);
                vx = v[0];
                vy = v[1];
                vz = v[2];
            }
            if (n_colliders > 0) {
                // MPM <-> rigid (legacy_coupler.py:385-397), before the boundary; the node
                // mass without the 1e3 particle-volume scale (legacy_coupler.py:375)
                const float p[3] = {px, py, pz};
                float v[3] = {vx, vy, vz};
                const float mreal = mm.w * 1e-3f;
                for (int k = 0; k < n_colliders; ++k) {  // MPM <-> Tool (legacy_coupler.py:381-383)
                    if (colliders[k].instance != e.x || colliders[k].kind != MPM_COLLIDER_TOOL) continue;
                    collide_tool(colliders[k], sdf_voxels, I.eps, I.dt, p, v);
                }
                for (int k = 0; k < n_colliders; ++k) {
                    if (colliders[k].instance != e.x || colliders[k].kind == MPM_COLLIDER_TOOL) continue;
                    collide_rigid(colliders[k], sdf_voxels, I.eps, I.dt, mreal, p, v,
                                  collider_force ? collider_force + 6 * k : nullptr);
                }
                vx = v[0];
                vy = v[1];
                vz = v[2];
            }
            vx = bc_vel(px, vx, I.bnd_lo[0], I.bnd_hi[0]);
            vy = bc_vel(py, vy, I.bnd_lo[1], I.bnd_hi[1]);
            vz = bc_vel(pz, vz, I.bnd_lo[2], I.bnd_hi[2]);
        }
        w.gv[g] = make_float4(vx, vy, vz, vz);  // w: a copy of z for the packed gather
        w.mm[g] = make_float4(0.f, 0.f, 0.f, 0.f);
        if (ln == 0) w.flag[I.blk_base + lb] = 0u;
    }
    // the last CTA to finish resets the active-block count for the next p2g: every CTA read
    // the count into registers before this barrier, so no fence is needed; no CTA waits on
    // another
    __syncthreads();
    if (threadIdx.x == 0) {
        if (atomicAdd(&w.counters[CNT_DONE], 1u) == gridDim.x - 1) {
            w.counters[CNT_ACTIVE] = 0u;
            w.counters[CNT_DONE] = 0u;
            if (count_op) w.counters[CNT_GRID_OPS] = ops + 1u;
        }
    }
}

// ---------------------------------------------------------------- state I/O

__global__ void k_get_state(mpm_problem prob, mpm_particles par, float* pos, float* vel, float* C, float* F, float* Jp,
                            uint8_t* active) {
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= prob.n_particles) return;
    const int g = par.gid[s];
    const int64_t st = par.state_stride;
    for (int d = 0; d < 3; ++d) {
        if (pos) pos[(int64_t)g * 3 + d] = par.state[(MPM_CH_X + d) * st + s];
        if (vel) vel[(int64_t)g * 3 + d] = par.state[(MPM_CH_V + d) * st + s];
    }
    for (int k = 0; k < 9; ++k) {
        if (C) C[(int64_t)g * 9 + k] = par.state[(MPM_CH_C + k) * st + s];
        if (F) F[(int64_t)g * 9 + k] = par.state[(MPM_CH_F + k) * st + s];
    }
    if (Jp) Jp[g] = par.state[MPM_CH_JP * st + s];
    if (active) active[g] = (par.pflags[s] & MPM_PFLAG_ACTIVE) ? 1 : 0;
}

__global__ void k_set_state(mpm_problem prob, mpm_particles par, const float* pos, const float* vel, const float* C,
                            const float* F, const float* Jp, const uint8_t* active) {
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= prob.n_particles) return;
    const int g = par.gid[s];
    const int64_t st = par.state_stride;
    for (int d = 0; d < 3; ++d) {
        if (pos) par.state[(MPM_CH_X + d) * st + s] = pos[(int64_t)g * 3 + d];
        if (vel) par.state[(MPM_CH_V + d) * st + s] = vel[(int64_t)g * 3 + d];
    }
    for (int k = 0; k < 9; ++k) {
        if (C) par.state[(MPM_CH_C + k) * st + s] = C[(int64_t)g * 9 + k];
        if (F) par.state[(MPM_CH_F + k) * st + s] = F[(int64_t)g * 9 + k];
    }
    if (Jp) par.state[MPM_CH_JP * st + s] = Jp[g];
    if (active) par.pflags[s] = (uint8_t)((par.pflags[s] & ~MPM_PFLAG_ACTIVE) | (active[g] ? MPM_PFLAG_ACTIVE : 0));
}

__global__ void k_set_pos(mpm_problem prob, const mpm_instance* __restrict__ inst, const mpm_material* __restrict__ mats,
                          mpm_particles par, int n, const int* idx, const float* pos) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const int g = idx[i];
    if (g < 0 || g >= prob.n_particles) return;
    const int s = par.slot[g];
    const int64_t st = par.state_stride;
    const int k = find_instance_by_particle(inst, prob.n_instances, s);
    const float djp = mats[inst[k].mat_base + par.mat[s]].default_Jp;
    for (int d = 0; d < 3; ++d) {
        par.state[(MPM_CH_X + d) * st + s] = pos[(int64_t)i * 3 + d];
        par.state[(MPM_CH_V + d) * st + s] = 0.f;
    }
    for (int kk = 0; kk < 9; ++kk) {
        par.state[(MPM_CH_C + kk) * st + s] = 0.f;
        par.state[(MPM_CH_F + kk) * st + s] = (kk % 4 == 0) ? 1.f : 0.f;
    }
    par.state[MPM_CH_JP * st + s] = djp;
}

__global__ void k_set_vel(mpm_problem prob, mpm_particles par, int n, const int* idx, const float* vel) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const int g = idx[i];
    if (g < 0 || g >= prob.n_particles) return;
    const int s = par.slot[g];
    for (int d = 0; d < 3; ++d) par.state[(MPM_CH_V + d) * par.state_stride + s] = vel[(int64_t)i * 3 + d];
}

__global__ void k_set_flag(mpm_problem prob, mpm_particles par, int n, const int* idx, const uint8_t* val, uint8_t bit) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const int g = idx[i];
    if (g < 0 || g >= prob.n_particles) return;
    const int s = par.slot[g];
    par.pflags[s] = (uint8_t)((par.pflags[s] & ~bit) | (val[i] ? bit : 0));
}

#include "mpm_adjoint.cuh"

// ---------------------------------------------------------------- host side

struct DevInfo {
    int sms = 0;
    int occ_p2g[3] = {0, 0, 0};
    int occ_g2p[3] = {0, 0, 0};
    int occ_g2p2g[3] = {0, 0, 0};
    int occ_grid = 0;
};

static std::mutex g_mu;
static DevInfo g_dev[64];

template <int P, typename K>
static int occ_of(K k) {
    int n = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, k, P, 0);
    return n > 0 ? n : 1;
}

static const DevInfo* dev_info() {
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return nullptr;
    std::lock_guard<std::mutex> lk(g_mu);
    DevInfo& d = g_dev[dev];
    if (d.sms == 0) {
        int sms = 0;
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        d.occ_p2g[0] = occ_of<128>(k_p2g<128, false, false>);
        d.occ_p2g[1] = occ_of<256>(k_p2g<256, false, false>);
        d.occ_p2g[2] = occ_of<512>(k_p2g<512, false, false>);
        d.occ_g2p[0] = occ_of<128>(k_g2p<128, false>);
        d.occ_g2p[1] = occ_of<256>(k_g2p<256, false>);
        d.occ_g2p[2] = occ_of<512>(k_g2p<512, false>);
        d.occ_g2p2g[0] = occ_of<128>(k_g2p2g<128, false, false>);
        d.occ_g2p2g[1] = occ_of<256>(k_g2p2g<256, false, false>);
        d.occ_g2p2g[2] = occ_of<512>(k_g2p2g<512, false, false>);
        int n = 0;
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, k_grid_op<false>, 256, 0);
        d.occ_grid = n > 0 ? n : 1;
        d.sms = sms > 0 ? sms : 1;
    }
    return &d;
}

static int p_index(int P) { return P == 128 ? 0 : (P == 256 ? 1 : (P == 512 ? 2 : -1)); }

static int check_problem(const mpm_problem* p) {
    if (!p) return MPM_E_INVALID;
    if (p->n_instances <= 0 || p->n_particles < 0 || p->n_blocks <= 0 || p->n_materials <= 0) return MPM_E_INVALID;
    if (p_index(p->chunk_particles) < 0) return MPM_E_INVALID;
    if (p->n_blocks > MAX_BLOCKS || p->n_blocks > INT32_MAX) return MPM_E_CAPACITY;
    int32_t need = 0;
    mpm_max_chunks(p->n_particles, p->n_blocks, p->chunk_particles, &need);
    if (p->max_chunks < need) return MPM_E_INVALID;
    return MPM_OK;
}

static int check_par(const mpm_problem* p, const mpm_particles* par) {
    if (!par || !par->state || !par->mat || !par->pflags || !par->gid || !par->slot) return MPM_E_INVALID;
    if (par->state_stride < p->n_particles) return MPM_E_INVALID;
    if ((par->mu_p == nullptr) != (par->lam_p == nullptr)) return MPM_E_INVALID;
    if ((par->actu == nullptr) != (par->muscle_dir == nullptr)) return MPM_E_INVALID;
    return MPM_OK;
}

static inline int cuda_ok() {
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) {
        fprintf(stderr, "genesis_b200_mpm: CUDA error %s\n", cudaGetErrorString(e));
        return MPM_E_CUDA;
    }
    return MPM_OK;
}

static int launch_sort(const mpm_problem* prob, const mpm_tables* tab, mpm_particles* par, void* ws, cudaStream_t s) {
    Ws w = ws_of(*prob, ws);
    const int64_t nb = prob->n_blocks;
    if (cudaMemsetAsync(w.bin_count, 0, nb * sizeof(int), s) != cudaSuccess) return MPM_E_CUDA;
    const int n = prob->n_particles;
    const int T = 256;
    if (n > 0) k_sort_keys<<<(n + T - 1) / T, T, 0, s>>>(*prob, tab->instances, *par, w);
    const int ntiles = (int)((nb + SCAN_TILE - 1) / SCAN_TILE);
    k_scan_reduce<<<ntiles, SCAN_T, 0, s>>>(nb, prob->chunk_particles, w);
    k_scan_tiles<<<1, SCAN_T, 0, s>>>(ntiles, w);
    k_scan_apply<<<ntiles, SCAN_T, 0, s>>>(nb, prob->chunk_particles, w);
    k_build_chunks<<<(int)((nb + T - 1) / T), T, 0, s>>>(*prob, tab->instances, w);
    if (n > 0) {
        k_sort_scatter<<<(n + T - 1) / T, T, 0, s>>>(*prob, *par, w);
        const DevInfo* d = dev_info();
        if (!d) return MPM_E_CUDA;
        const int P = prob->chunk_particles;
        int ctas = d->sms * (2048 / P);
        if (ctas > prob->max_chunks) ctas = prob->max_chunks > 0 ? prob->max_chunks : 1;
        if (P == 128)
            k_sort_interleave<128><<<ctas, 128, 0, s>>>(*prob, tab->instances, *par, w);
        else if (P == 256)
            k_sort_interleave<256><<<ctas, 256, 0, s>>>(*prob, tab->instances, *par, w);
        else
            k_sort_interleave<512><<<ctas, 512, 0, s>>>(*prob, tab->instances, *par, w);
    }
    return cuda_ok();
}

static int persistent_ctas(const mpm_problem* prob, int occ) {
    const DevInfo* d = dev_info();
    if (!d) return -1;
    int ctas = prob->grid_ctas > 0 ? prob->grid_ctas : d->sms * occ;
    if (ctas > prob->max_chunks) ctas = prob->max_chunks > 0 ? prob->max_chunks : 1;
    return ctas;
}

// launch helpers: one kernel per chunk size, muscle term and CPIC
template <int P>
static void run_p2g(bool m, bool cp, int ctas, cudaStream_t s, const P2GArgs& a) {
    if (m)
        cp ? k_p2g<P, true, true><<<ctas, P, 0, s>>>(a) : k_p2g<P, true, false><<<ctas, P, 0, s>>>(a);
    else
        cp ? k_p2g<P, false, true><<<ctas, P, 0, s>>>(a) : k_p2g<P, false, false><<<ctas, P, 0, s>>>(a);
}
template <int P>
static void run_g2p2g(bool m, bool cp, int ctas, cudaStream_t s, const P2GArgs& a) {
    if (m)
        cp ? k_g2p2g<P, true, true><<<ctas, P, 0, s>>>(a) : k_g2p2g<P, true, false><<<ctas, P, 0, s>>>(a);
    else
        cp ? k_g2p2g<P, false, true><<<ctas, P, 0, s>>>(a) : k_g2p2g<P, false, false><<<ctas, P, 0, s>>>(a);
}
template <int P>
static void run_g2p(bool cp, int ctas, cudaStream_t s, const P2GArgs& a) {
    cp ? k_g2p<P, true><<<ctas, P, 0, s>>>(a) : k_g2p<P, false><<<ctas, P, 0, s>>>(a);
}

// the kernels' arguments; CPIC runs when the problem asks for it and the instance has
// colliders (MPM_E_INVALID if its buffers are missing or there are more than 254 colliders,
// the limit of its one-byte node codes)
static int p2g_args(const mpm_problem* prob, const mpm_tables* tab, const mpm_particles* par, void* ws, P2GArgs& a,
                    bool& cpic) {
    const int nc = tab->colliders ? tab->n_colliders : 0;
    cpic = (prob->flags & MPM_PROBF_CPIC) && nc > 0;
    if (cpic && (!par->cpic_normal || !par->cpic_sep || nc > 254)) return MPM_E_INVALID;
    a = P2GArgs{*prob,           tab->instances, tab->materials,     *par,           ws_of(*prob, ws),
                tab->colliders, nc,             tab->collider_force, tab->sdf_voxels};
    return MPM_OK;
}

static int launch_p2g(const mpm_problem* prob, const mpm_tables* tab, mpm_particles* par, void* ws, cudaStream_t s) {
    const DevInfo* d = dev_info();
    if (!d) return MPM_E_CUDA;
    P2GArgs a;
    bool cpic;
    int rc = p2g_args(prob, tab, par, ws, a, cpic);
    if (rc) return rc;
    const int pi = p_index(prob->chunk_particles);
    const int ctas = persistent_ctas(prob, d->occ_p2g[pi]);
    const bool muscle = par->actu != nullptr;
    switch (prob->chunk_particles) {
        case 128: run_p2g<128>(muscle, cpic, ctas, s, a); break;
        case 256: run_p2g<256>(muscle, cpic, ctas, s, a); break;
        case 512: run_p2g<512>(muscle, cpic, ctas, s, a); break;
    }
    if ((prob->flags & MPM_PROBF_NONFREE) && prob->n_particles > 0)
        k_nonfree_zero<<<(prob->n_particles + 255) / 256, 256, 0, s>>>(*prob, tab->instances, *par, a.w);
    return cuda_ok();
}

// advance = false (the adjoint's recompute): the colliders keep their pose and accumulate no force
static int launch_grid_op(const mpm_problem* prob, const mpm_tables* tab, void* ws, cudaStream_t s,
                          bool advance = true) {
    const DevInfo* d = dev_info();
    if (!d) return MPM_E_CUDA;
    int ctas = prob->grid_ctas > 0 ? prob->grid_ctas : d->sms * d->occ_grid;
    const int64_t need = (prob->n_blocks + 3) / 4;
    if (ctas > need) ctas = (int)need;
    if (tab->n_colliders < 0) return MPM_E_INVALID;
    const int nc = tab->colliders ? tab->n_colliders : 0;
    if (tab->n_force_fields < 0 || (tab->n_force_fields > 0 && !tab->force_fields)) return MPM_E_INVALID;
    const int nff = tab->force_fields ? tab->n_force_fields : 0;
    if (nff > 0)
        k_grid_op<true><<<ctas, 256, 0, s>>>(*prob, tab->instances, ws_of(*prob, ws), tab->colliders, nc,
                                              advance ? tab->collider_force : nullptr, tab->sdf_voxels,
                                              tab->force_fields, nff, tab->ff_perm, advance ? 1 : 0);
    else
        k_grid_op<false><<<ctas, 256, 0, s>>>(*prob, tab->instances, ws_of(*prob, ws), tab->colliders, nc,
                                               advance ? tab->collider_force : nullptr, tab->sdf_voxels, nullptr, 0,
                                               nullptr, advance ? 1 : 0);
    if (nc > 0 && advance)
        k_advance_colliders<<<(nc + 63) / 64, 64, 0, s>>>(tab->instances, prob->n_instances, tab->colliders, nc);
    return cuda_ok();
}

static int launch_g2p(const mpm_problem* prob, const mpm_tables* tab, mpm_particles* par, void* ws, cudaStream_t s) {
    const DevInfo* d = dev_info();
    if (!d) return MPM_E_CUDA;
    P2GArgs a;
    bool cpic;
    int rc = p2g_args(prob, tab, par, ws, a, cpic);
    if (rc) return rc;
    const int pi = p_index(prob->chunk_particles);
    const int ctas = persistent_ctas(prob, d->occ_g2p[pi]);
    switch (prob->chunk_particles) {
        case 128: run_g2p<128>(cpic, ctas, s, a); break;
        case 256: run_g2p<256>(cpic, ctas, s, a); break;
        case 512: run_g2p<512>(cpic, ctas, s, a); break;
    }
    return cuda_ok();
}

static int launch_g2p2g(const mpm_problem* prob, const mpm_tables* tab, mpm_particles* par, void* ws,
                        cudaStream_t s) {
    const DevInfo* d = dev_info();
    if (!d) return MPM_E_CUDA;
    P2GArgs a;
    bool cpic;
    int rc = p2g_args(prob, tab, par, ws, a, cpic);
    if (rc) return rc;
    const int pi = p_index(prob->chunk_particles);
    const int ctas = persistent_ctas(prob, d->occ_g2p2g[pi]);
    const bool muscle = par->actu != nullptr;
    switch (prob->chunk_particles) {
        case 128: run_g2p2g<128>(muscle, cpic, ctas, s, a); break;
        case 256: run_g2p2g<256>(muscle, cpic, ctas, s, a); break;
        case 512: run_g2p2g<512>(muscle, cpic, ctas, s, a); break;
    }
    if ((prob->flags & MPM_PROBF_NONFREE) && prob->n_particles > 0)
        k_nonfree_zero<<<(prob->n_particles + 255) / 256, 256, 0, s>>>(*prob, tab->instances, *par, a.w);
    return cuda_ok();
}

}  // namespace gbm

using namespace gbm;

// ---------------------------------------------------------------- tool SDF voxels
// compute_sdf_data (utils/mesh.py:179-201): the signed distance of every voxel centre of a
// res^3 lattice over [-radius, radius]^3 to a triangle mesh.  Each CTA stages the mesh in
// tiles of 256 triangles in shared memory; every thread owns one voxel and keeps the nearest
// squared distance and the winding number.

// squared distance from p to triangle (a, b, c): the closest point by the Voronoi region of
// p (Ericson, Real-Time Collision Detection, 5.1.5)
__device__ __forceinline__ float tri_dist2(const float* p, const float* a, const float* b, const float* c) {
    float ab[3], ac[3], ap[3];
#pragma unroll
    for (int i = 0; i < 3; ++i) {
        ab[i] = b[i] - a[i];
        ac[i] = c[i] - a[i];
        ap[i] = p[i] - a[i];
    }
    auto dot = [](const float* u, const float* v) { return u[0] * v[0] + u[1] * v[1] + u[2] * v[2]; };
    float q[3];
    const float d1 = dot(ab, ap), d2 = dot(ac, ap);
    if (d1 <= 0.f && d2 <= 0.f) {
        q[0] = a[0], q[1] = a[1], q[2] = a[2];
    } else {
        float bp[3], cp[3];
#pragma unroll
        for (int i = 0; i < 3; ++i) {
            bp[i] = p[i] - b[i];
            cp[i] = p[i] - c[i];
        }
        const float d3 = dot(ab, bp), d4 = dot(ac, bp), d5 = dot(ab, cp), d6 = dot(ac, cp);
        const float vc = d1 * d4 - d3 * d2, vb = d5 * d2 - d1 * d6, va = d3 * d6 - d5 * d4;
        if (d3 >= 0.f && d4 <= d3) {
            q[0] = b[0], q[1] = b[1], q[2] = b[2];
        } else if (d6 >= 0.f && d5 <= d6) {
            q[0] = c[0], q[1] = c[1], q[2] = c[2];
        } else if (vc <= 0.f && d1 >= 0.f && d3 <= 0.f) {
            const float t = d1 / (d1 - d3);
#pragma unroll
            for (int i = 0; i < 3; ++i) q[i] = a[i] + t * ab[i];
        } else if (vb <= 0.f && d2 >= 0.f && d6 <= 0.f) {
            const float t = d2 / (d2 - d6);
#pragma unroll
            for (int i = 0; i < 3; ++i) q[i] = a[i] + t * ac[i];
        } else if (va <= 0.f && (d4 - d3) >= 0.f && (d5 - d6) >= 0.f) {
            const float t = (d4 - d3) / ((d4 - d3) + (d5 - d6));
#pragma unroll
            for (int i = 0; i < 3; ++i) q[i] = b[i] + t * (c[i] - b[i]);
        } else {
            const float den = 1.f / (va + vb + vc);
            const float v = vb * den, w = vc * den;
#pragma unroll
            for (int i = 0; i < 3; ++i) q[i] = a[i] + ab[i] * v + ac[i] * w;
        }
    }
    const float d[3] = {p[0] - q[0], p[1] - q[1], p[2] - q[2]};
    return d[0] * d[0] + d[1] * d[1] + d[2] * d[2];
}

// solid angle of triangle (a, b, c) seen from p, signed by the triangle's orientation
// (Van Oosterom & Strackee 1983): tan(omega / 2) = det[r_a r_b r_c] /
// (|r_a||r_b||r_c| + (r_a.r_b)|r_c| + (r_a.r_c)|r_b| + (r_b.r_c)|r_a|)
__device__ __forceinline__ float tri_solid_angle(const float* p, const float* a, const float* b, const float* c) {
    const float ra[3] = {a[0] - p[0], a[1] - p[1], a[2] - p[2]};
    const float rb[3] = {b[0] - p[0], b[1] - p[1], b[2] - p[2]};
    const float rc[3] = {c[0] - p[0], c[1] - p[1], c[2] - p[2]};
    const float la = sqrtf(ra[0] * ra[0] + ra[1] * ra[1] + ra[2] * ra[2]);
    const float lb = sqrtf(rb[0] * rb[0] + rb[1] * rb[1] + rb[2] * rb[2]);
    const float lc = sqrtf(rc[0] * rc[0] + rc[1] * rc[1] + rc[2] * rc[2]);
    const float det = ra[0] * (rb[1] * rc[2] - rb[2] * rc[1]) - ra[1] * (rb[0] * rc[2] - rb[2] * rc[0]) +
                      ra[2] * (rb[0] * rc[1] - rb[1] * rc[0]);
    const float den = la * lb * lc + (ra[0] * rb[0] + ra[1] * rb[1] + ra[2] * rb[2]) * lc +
                      (ra[0] * rc[0] + ra[1] * rc[1] + ra[2] * rc[2]) * lb +
                      (rb[0] * rc[0] + rb[1] * rc[1] + rb[2] * rc[2]) * la;
    return 2.f * atan2f(det, den);
}

constexpr int SDF_T = 256;

// Signed distance of a closed triangle mesh at the nodes of an axis-aligned grid (node (i, j, k)
// at origin + (i, j, k) * step, x-major): the nearest-triangle distance, negative where the
// generalised winding number exceeds 1/2.  Faces are staged through shared memory SDF_T at a time.
struct SdfGrid {
    float origin[3];
    float step[3];
    int res[3];
};

__global__ void __launch_bounds__(SDF_T) k_sdf_grid(const float* __restrict__ V, int nv, const int* __restrict__ Fc,
                                                    int nf, SdfGrid G, float* __restrict__ out) {
    __shared__ float tri[SDF_T][9];
    const int64_t n = (int64_t)G.res[0] * G.res[1] * G.res[2];
    const int64_t vid = (int64_t)blockIdx.x * SDF_T + threadIdx.x;
    const int i = (int)(vid / ((int64_t)G.res[1] * G.res[2])), j = (int)((vid / G.res[2]) % G.res[1]),
              k = (int)(vid % G.res[2]);
    const float p[3] = {G.origin[0] + G.step[0] * (float)i, G.origin[1] + G.step[1] * (float)j,
                        G.origin[2] + G.step[2] * (float)k};
    float d2 = 3.402823466e38f, wind = 0.f;
    for (int f0 = 0; f0 < nf; f0 += SDF_T) {
        const int f = f0 + threadIdx.x;
        bool ok = false;
        if (f < nf) {
            const int ia = Fc[3 * f], ib = Fc[3 * f + 1], ic = Fc[3 * f + 2];
            ok = ia >= 0 && ib >= 0 && ic >= 0 && ia < nv && ib < nv && ic < nv;
            if (ok) {
#pragma unroll
                for (int d = 0; d < 3; ++d) {
                    tri[threadIdx.x][d] = V[3 * ia + d];
                    tri[threadIdx.x][3 + d] = V[3 * ib + d];
                    tri[threadIdx.x][6 + d] = V[3 * ic + d];
                }
            }
        }
        if (!ok) {  // a padding (or invalid) face: degenerate, far away, no solid angle
#pragma unroll
            for (int d = 0; d < 9; ++d) tri[threadIdx.x][d] = 1e18f;
        }
        __syncthreads();
        const int m = min(SDF_T, nf - f0);
        if (vid < n) {
            for (int t = 0; t < m; ++t) {
                const float* T = tri[t];
                if (T[0] == 1e18f) continue;
                d2 = fminf(d2, tri_dist2(p, T, T + 3, T + 6));
                wind += tri_solid_angle(p, T, T + 3, T + 6);
            }
        }
        __syncthreads();
    }
    if (vid < n) {
        const float w = wind * (1.f / (4.f * 3.14159265358979f));
        out[vid] = (fabsf(w) > 0.5f ? -1.f : 1.f) * sqrtf(d2);
    }
}

extern "C" {

int mpm_abi_version(void) { return MPM_ABI_VERSION; }

int mpm_struct_sizes(int32_t* out7) {
    if (!out7) return MPM_E_INVALID;
    out7[0] = (int32_t)sizeof(mpm_instance);
    out7[1] = (int32_t)sizeof(mpm_material);
    out7[2] = (int32_t)sizeof(mpm_problem);
    out7[3] = (int32_t)sizeof(mpm_particles);
    out7[4] = (int32_t)sizeof(mpm_tables);
    out7[5] = (int32_t)sizeof(mpm_collider);
    out7[6] = (int32_t)sizeof(mpm_force_field);
    return MPM_OK;
}

int mpm_max_chunks(int32_t n_particles, int64_t n_blocks, int32_t chunk_particles, int32_t* out) {
    if (!out || chunk_particles <= 0 || n_particles < 0 || n_blocks < 0) return MPM_E_INVALID;
    int64_t m = (int64_t)n_particles / chunk_particles + (n_particles < n_blocks ? n_particles : n_blocks) + 1;
    if (m > INT32_MAX) return MPM_E_CAPACITY;
    *out = (int32_t)m;
    return MPM_OK;
}

int mpm_workspace_bytes(const mpm_problem* prob, uint64_t* out) {
    int rc = check_problem(prob);
    if (rc) return rc;
    if (!out) return MPM_E_INVALID;
    *out = layout_of(*prob).total;
    return MPM_OK;
}

int mpm_grid_offsets(const mpm_problem* prob, uint64_t* mm_offset, uint64_t* vel_offset) {
    int rc = check_problem(prob);
    if (rc) return rc;
    if (!mm_offset || !vel_offset) return MPM_E_INVALID;
    Layout L = layout_of(*prob);
    *mm_offset = L.off[0];
    *vel_offset = L.off[1];
    return MPM_OK;
}

int mpm_workspace_init(const mpm_problem* prob, void* workspace, void* stream) {
    int rc = check_problem(prob);
    if (rc) return rc;
    if (!workspace) return MPM_E_INVALID;
    // Only what is read before it is written needs zeros: the grids (mm accumulates; gv of
    // blocks no particle reached is read as zero velocity), the block flags, the counters
    // and the per-instance statuses.  The sort scratch between them (keys, ranks, chunk
    // table, permutation arrays: ~110 B per particle) is always written first.
    const Layout L = layout_of(*prob);
    cudaStream_t s = (cudaStream_t)stream;
    unsigned char* b = (unsigned char*)workspace;
    if (cudaMemsetAsync(b, 0, L.off[3], s) != cudaSuccess) return MPM_E_CUDA;  // mm, gv, flag
    if (cudaMemsetAsync(b + L.off[17], 0, L.total - L.off[17], s) != cudaSuccess) return MPM_E_CUDA;
    return MPM_OK;
}

int mpm_sort_particles(const mpm_problem* prob, const mpm_tables* tab, mpm_particles* par, void* workspace,
                       void* stream) {
    int rc = check_problem(prob);
    if (rc) return rc;
    if ((rc = check_par(prob, par))) return rc;
    if (!tab || !tab->instances || !workspace) return MPM_E_INVALID;
    return launch_sort(prob, tab, par, workspace, (cudaStream_t)stream);
}

int mpm_p2g(const mpm_problem* prob, const mpm_tables* tab, mpm_particles* par, void* workspace, void* stream) {
    int rc = check_problem(prob);
    if (rc) return rc;
    if ((rc = check_par(prob, par))) return rc;
    if (!tab || !tab->instances || !tab->materials || !workspace) return MPM_E_INVALID;
    return launch_p2g(prob, tab, par, workspace, (cudaStream_t)stream);
}

int mpm_grid_op(const mpm_problem* prob, const mpm_tables* tab, void* workspace, void* stream) {
    int rc = check_problem(prob);
    if (rc) return rc;
    if (!tab || !tab->instances || !workspace) return MPM_E_INVALID;
    return launch_grid_op(prob, tab, workspace, (cudaStream_t)stream);
}

int mpm_g2p(const mpm_problem* prob, const mpm_tables* tab, mpm_particles* par, void* workspace, void* stream) {
    int rc = check_problem(prob);
    if (rc) return rc;
    if ((rc = check_par(prob, par))) return rc;
    if (!tab || !tab->instances || !workspace) return MPM_E_INVALID;
    return launch_g2p(prob, tab, par, workspace, (cudaStream_t)stream);
}

// Optional per-launch timing of substeps_impl (mpm_substeps_profile): an event is recorded
// after every launch group, so the time between consecutive events belongs to that group's
// kernel kind and the kinds' times add up to the whole run.
struct Prof {
    static constexpr int MAX_EV = 4096;
    cudaEvent_t ev[MAX_EV];
    int kind[MAX_EV];
    int n = 0;
    bool ok = true;
    cudaStream_t s;
    explicit Prof(cudaStream_t st) : s(st) {
        ok = cudaEventCreate(&ev[0]) == cudaSuccess && cudaEventRecord(ev[0], s) == cudaSuccess;
        n = ok ? 1 : 0;
    }
    void mark(int k) {
        if (!ok || n >= MAX_EV) {
            ok = false;
            return;
        }
        if (cudaEventCreate(&ev[n]) != cudaSuccess || cudaEventRecord(ev[n], s) != cudaSuccess) {
            ok = false;
            return;
        }
        kind[n++] = k;
    }
    ~Prof() {
        for (int i = 0; i < n; ++i) cudaEventDestroy(ev[i]);
    }
};

// n substeps.  The first substep starts with p2g; between substeps the g2p of substep i
// and the p2g of substep i+1 run fused unless a re-sort falls between them, in which case
// g2p, sort and p2g run separately; the last substep ends with g2p, so x, v, C, F, Jp are
// all materialised when the call returns.
static int substeps_impl(const mpm_problem* prob, const mpm_tables* tab, mpm_particles* par, void* ws, int32_t n,
                         int32_t sort_interval, int64_t first, cudaStream_t s, Prof* pr = nullptr) {
    if (n <= 0) return MPM_OK;
    int rc;
    auto mark = [&](int k) {
        if (pr) pr->mark(k);
    };
    auto sort_due = [&](int32_t i) { return sort_interval > 0 && ((first + i) % sort_interval) == 0; };
    if (sort_due(0)) {
        if ((rc = launch_sort(prob, tab, par, ws, s))) return rc;
        mark(MPM_KIND_SORT);
    }
    if ((rc = launch_p2g(prob, tab, par, ws, s))) return rc;
    mark(MPM_KIND_P2G);
    if ((rc = launch_grid_op(prob, tab, ws, s))) return rc;
    mark(MPM_KIND_GRID_OP);
    for (int32_t i = 1; i < n; ++i) {
        if (sort_due(i)) {
            if ((rc = launch_g2p(prob, tab, par, ws, s))) return rc;
            mark(MPM_KIND_G2P);
            if ((rc = launch_sort(prob, tab, par, ws, s))) return rc;
            mark(MPM_KIND_SORT);
            if ((rc = launch_p2g(prob, tab, par, ws, s))) return rc;
            mark(MPM_KIND_P2G);
        } else {
            if ((rc = launch_g2p2g(prob, tab, par, ws, s))) return rc;
            mark(MPM_KIND_G2P2G);
        }
        if ((rc = launch_grid_op(prob, tab, ws, s))) return rc;
        mark(MPM_KIND_GRID_OP);
    }
    if ((rc = launch_g2p(prob, tab, par, ws, s))) return rc;
    mark(MPM_KIND_G2P);
    return MPM_OK;
}

int mpm_substeps_profile(const mpm_problem* prob, const mpm_tables* tab, mpm_particles* par, void* workspace,
                         int32_t n_substeps, int32_t sort_interval, int64_t first_substep, float* ms_by_kind,
                         int32_t* launches_by_kind, void* stream) {
    int rc = check_problem(prob);
    if (rc) return rc;
    if ((rc = check_par(prob, par))) return rc;
    if (!tab || !tab->instances || !tab->materials || !workspace || n_substeps < 0 || !ms_by_kind ||
        !launches_by_kind)
        return MPM_E_INVALID;
    cudaStream_t s = (cudaStream_t)stream;
    for (int k = 0; k < MPM_N_KINDS; ++k) {
        ms_by_kind[k] = 0.f;
        launches_by_kind[k] = 0;
    }
    Prof pr(s);
    if (!pr.ok) return MPM_E_CUDA;
    rc = substeps_impl(prob, tab, par, workspace, n_substeps, sort_interval, first_substep, s, &pr);
    if (rc) return rc;
    if (!pr.ok) return MPM_E_CAPACITY;  // more launches than the profiler's events
    if (cudaStreamSynchronize(s) != cudaSuccess) return MPM_E_CUDA;
    for (int i = 1; i < pr.n; ++i) {
        float ms = 0.f;
        if (cudaEventElapsedTime(&ms, pr.ev[i - 1], pr.ev[i]) != cudaSuccess) return MPM_E_CUDA;
        ms_by_kind[pr.kind[i]] += ms;
        // a sort is 7 kernels (keys, 3 scan passes, chunk table, scatter, lane deal), 4 without particles
        launches_by_kind[pr.kind[i]] += pr.kind[i] == MPM_KIND_SORT ? (prob->n_particles > 0 ? 7 : 4) : 1;
    }
    return MPM_OK;
}

int mpm_g2p2g(const mpm_problem* prob, const mpm_tables* tab, mpm_particles* par, void* workspace, void* stream) {
    int rc = check_problem(prob);
    if (rc) return rc;
    if ((rc = check_par(prob, par))) return rc;
    if (!tab || !tab->instances || !tab->materials || !workspace) return MPM_E_INVALID;
    return launch_g2p2g(prob, tab, par, workspace, (cudaStream_t)stream);
}

int mpm_substeps(const mpm_problem* prob, const mpm_tables* tab, mpm_particles* par, void* workspace,
                 int32_t n_substeps, int32_t sort_interval, int64_t first_substep, void* stream) {
    int rc = check_problem(prob);
    if (rc) return rc;
    if ((rc = check_par(prob, par))) return rc;
    if (!tab || !tab->instances || !tab->materials || !workspace || n_substeps < 0) return MPM_E_INVALID;
    return substeps_impl(prob, tab, par, workspace, n_substeps, sort_interval, first_substep, (cudaStream_t)stream);
}

// ---------------------------------------------------------------- allocation-free variant
// Scratch for mpm_substeps_noalloc.  It lives in the module's static device memory, so a
// caller that may not allocate (a plugin host that forbids cudaMalloc, a pre-reserved
// memory pool, code running inside another runtime's allocator) still gets the full
// substep.  Every GPU that loads this library holds these bytes until the process exits.
static __device__ __align__(256) unsigned char g_noalloc_scratch[MPM_NOALLOC_SCRATCH_BYTES];

static std::mutex g_noalloc_mu;
static void* g_noalloc_ptr[64];

// Device address of the scratch array on the current device.  In host code the array's
// name is only a host-side stand-in, so the address must come from cudaGetSymbolAddress,
// asked with that device current.  Outside stream capture the address is asked again on
// every call, so a context torn down and rebuilt (cudaDeviceReset) is followed to the
// module's new address; while `s` is capturing, the address cached by an earlier call
// is used (the first call on a device must therefore come before any capture).
static int noalloc_scratch(cudaStream_t s, void** out) {
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return MPM_E_CUDA;
    cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
    if (cudaStreamIsCapturing(s, &cap) != cudaSuccess) {
        cudaGetLastError();
        return MPM_E_CUDA;
    }
    std::lock_guard<std::mutex> lk(g_noalloc_mu);
    if (!g_noalloc_ptr[dev] || cap == cudaStreamCaptureStatusNone) {
        if (cap != cudaStreamCaptureStatusNone) return MPM_E_INVALID;  // no set-up inside a capture
        void* p = nullptr;
        if (cudaGetSymbolAddress(&p, g_noalloc_scratch) != cudaSuccess || !p) {
            cudaGetLastError();
            return MPM_E_CUDA;
        }
        g_noalloc_ptr[dev] = p;
    }
    *out = g_noalloc_ptr[dev];
    return MPM_OK;
}

int mpm_substeps_noalloc(const mpm_problem* prob, const mpm_tables* tab, mpm_particles* par, int32_t n_substeps,
                         int32_t sort_interval, int64_t first_substep, void* stream) {
    int rc = check_problem(prob);
    if (rc) return rc;
    if ((rc = check_par(prob, par))) return rc;
    if (!tab || !tab->instances || !tab->materials || n_substeps < 0) return MPM_E_INVALID;
    const uint64_t need = layout_of(*prob).total;
    if (need > (uint64_t)MPM_NOALLOC_SCRATCH_BYTES) return MPM_E_CAPACITY;
    cudaStream_t s = (cudaStream_t)stream;
    void* ws = nullptr;
    if ((rc = noalloc_scratch(s, &ws))) return rc;
    // the array keeps the previous call's contents (possibly another problem's layout):
    // start from the zeroed state mpm_workspace_init gives, then bin the particles
    if (cudaMemsetAsync(ws, 0, need, s) != cudaSuccess) return MPM_E_CUDA;
    if (n_substeps == 0) return MPM_OK;
    const bool sorts_first = sort_interval > 0 && (first_substep % sort_interval) == 0;
    if (!sorts_first && (rc = launch_sort(prob, tab, par, ws, s))) return rc;
    return substeps_impl(prob, tab, par, ws, n_substeps, sort_interval, first_substep, s);
}

int mpm_noalloc_status(const mpm_problem* prob, int32_t clear, uint32_t* out, uint32_t* inst_out, void* stream) {
    int rc = check_problem(prob);
    if (rc) return rc;
    if (!out) return MPM_E_INVALID;
    if (layout_of(*prob).total > (uint64_t)MPM_NOALLOC_SCRATCH_BYTES) return MPM_E_CAPACITY;
    cudaStream_t s = (cudaStream_t)stream;
    void* ws = nullptr;
    if ((rc = noalloc_scratch(s, &ws))) return rc;
    Ws w = ws_of(*prob, ws);
    const size_t ibytes = (size_t)prob->n_instances * 4;
    uint32_t v = 0;
    if (cudaMemcpyAsync(&v, &w.counters[CNT_STATUS], 4, cudaMemcpyDeviceToHost, s) != cudaSuccess) return MPM_E_CUDA;
    if (inst_out && ibytes &&
        cudaMemcpyAsync(inst_out, w.inst_status, ibytes, cudaMemcpyDeviceToHost, s) != cudaSuccess)
        return MPM_E_CUDA;
    if (cudaStreamSynchronize(s) != cudaSuccess) return MPM_E_CUDA;
    if (clear) {
        if (cudaMemsetAsync(&w.counters[CNT_STATUS], 0, 4, s) != cudaSuccess) return MPM_E_CUDA;
        if (ibytes && cudaMemsetAsync(w.inst_status, 0, ibytes, s) != cudaSuccess) return MPM_E_CUDA;
    }
    *out = v;
    return MPM_OK;
}

// ---------------------------------------------------------------- adjoint
int mpm_adjoint_workspace_bytes(const mpm_problem* prob, uint64_t* out) {
    int rc = check_problem(prob);
    if (rc) return rc;
    if (!out) return MPM_E_INVALID;
    uint64_t off[5];
    *out = adj_layout(*prob, off);
    return MPM_OK;
}

int mpm_substep_adjoint_colliders(const mpm_problem* prob, const mpm_tables* tab, const mpm_particles* state,
                                  float* adj, float* lame_bar, float* collider_bar, void* workspace,
                                  void* adj_workspace, void* stream) {
    int rc = check_problem(prob);
    if (rc) return rc;
    if ((rc = check_par(prob, state))) return rc;
    if (!tab || !tab->instances || !tab->materials || !adj || !lame_bar || !workspace || !adj_workspace)
        return MPM_E_INVALID;
    const int nc = (tab->colliders && tab->n_colliders > 0) ? tab->n_colliders : 0;
    if (tab->n_colliders < 0) return MPM_E_INVALID;
    if (nc > 0 && (prob->flags & MPM_PROBF_CPIC)) return MPM_E_INVALID;  // no adjoint of the particle-level coupling
    cudaStream_t s = (cudaStream_t)stream;
    const int n = prob->n_particles;
    AdjWs aw = adj_ws_of(*prob, adj_workspace);
    Ws w = ws_of(*prob, workspace);
    // forward recompute of the substep's grid on a scratch copy (p2g writes F and Jp)
    if (n > 0 && cudaMemcpy2DAsync(aw.state, aw.stride * 4, state->state, state->state_stride * 4, (size_t)n * 4,
                                   MPM_STATE_CH, cudaMemcpyDeviceToDevice, s) != cudaSuccess)
        return MPM_E_CUDA;
    mpm_particles sp = *state;
    sp.state = aw.state;
    sp.state_stride = aw.stride;
    if ((rc = launch_p2g(prob, tab, &sp, workspace, s))) return rc;
    const size_t nodes = (size_t)prob->n_blocks * BLK3;
    if (cudaMemcpyAsync(aw.saved_mm, w.mm, nodes * 16, cudaMemcpyDeviceToDevice, s) != cudaSuccess) return MPM_E_CUDA;
    if ((rc = launch_grid_op(prob, tab, workspace, s, false))) return rc;
    if (cudaMemsetAsync(aw.vbar, 0, nodes * 16, s) != cudaSuccess) return MPM_E_CUDA;
    if (n > 0) {
        k_adj_g2p<<<(n + 127) / 128, 128, 0, s>>>(*prob, tab->instances, *state, adj, w, aw);
        k_adj_grid<<<(int)((nodes + 255) / 256), 256, 0, s>>>(*prob, tab->instances, w, aw, tab->colliders, nc,
                                                               tab->sdf_voxels, collider_bar, tab->force_fields,
                                                               tab->force_fields ? tab->n_force_fields : 0,
                                                               tab->ff_perm);
        k_adj_p2g<<<(n + 127) / 128, 128, 0, s>>>(*prob, tab->instances, tab->materials, *state, adj, lame_bar, aw);
    }
    return cuda_ok();
}

// One recorded substep of grid_rec: the momentum and mass after p2g and the velocity after
// the grid op (float4 per node each), then the active-block list the grid op walked and its
// length.
struct RecGrid {
    float4* mm;
    float4* gv;
    int2* active;
    uint32_t* n_active;
};

static uint64_t rec_grid_bytes(const mpm_problem& p) {
    const uint64_t nodes = (uint64_t)p.n_blocks * BLK3;
    return align_up(nodes * 32 + (uint64_t)p.n_blocks * 8 + 16, 256);
}

static RecGrid rec_grid_of(const mpm_problem& p, void* base, int32_t j) {
    char* b = (char*)base + (uint64_t)j * rec_grid_bytes(p);
    const uint64_t nodes = (uint64_t)p.n_blocks * BLK3;
    RecGrid r;
    r.mm = (float4*)b;
    r.gv = (float4*)(b + nodes * 16);
    r.active = (int2*)(b + nodes * 32);
    r.n_active = (uint32_t*)(b + nodes * 32 + (uint64_t)p.n_blocks * 8);
    return r;
}

// Record the p2g result of the active blocks: their list, its length and their momentum and
// mass (the grid op, which runs next, clears both behind itself).  One 64-thread group per
// block; the adjoint reads nothing outside the active blocks.
__device__ __forceinline__ int64_t block_of_entry(const mpm_instance* __restrict__ inst, int2 e) {
    const mpm_instance& I = inst[e.x];
    const BlockCoord bc = unpack_bc(e.y);
    return I.blk_base + local_block(I, bc.bx, bc.by, bc.bz);
}

__global__ void __launch_bounds__(256) k_record_p2g(const mpm_instance* __restrict__ inst, Ws w, RecGrid r) {
    const int n_active = (int)w.counters[CNT_ACTIVE];
    const int gpc = blockDim.x / BLK3, grp = threadIdx.x / BLK3, ln = threadIdx.x % BLK3;
    if (blockIdx.x == 0 && threadIdx.x == 0) *r.n_active = (uint32_t)n_active;
    for (int i = blockIdx.x * gpc + grp; i < n_active; i += gridDim.x * gpc) {
        const int2 e = w.active[i];
        if (ln == 0) r.active[i] = e;
        const int64_t blk = block_of_entry(inst, e);
        r.mm[blk * BLK3 + ln] = w.mm[blk * BLK3 + ln];
    }
}

// Record the grid op's velocity of the blocks k_record_p2g listed.
__global__ void __launch_bounds__(256) k_record_gv(const mpm_instance* __restrict__ inst, Ws w, RecGrid r) {
    const int n_active = (int)*r.n_active;
    const int gpc = blockDim.x / BLK3, grp = threadIdx.x / BLK3, ln = threadIdx.x % BLK3;
    for (int i = blockIdx.x * gpc + grp; i < n_active; i += gridDim.x * gpc) {
        const int64_t blk = block_of_entry(inst, r.active[i]);
        r.gv[blk * BLK3 + ln] = w.gv[blk * BLK3 + ln];
    }
}

int mpm_record_grid_bytes(const mpm_problem* prob, uint64_t* out) {
    int rc = check_problem(prob);
    if (rc) return rc;
    if (!out) return MPM_E_INVALID;
    *out = rec_grid_bytes(*prob);
    return MPM_OK;
}

int mpm_substeps_record(const mpm_problem* prob, const mpm_tables* tab, mpm_particles* par, void* workspace,
                        int32_t n_substeps, float* state_rec, void* grid_rec, void* stream) {
    int rc = check_problem(prob);
    if (rc) return rc;
    if ((rc = check_par(prob, par))) return rc;
    if (!tab || !tab->instances || !tab->materials || !workspace || n_substeps < 0) return MPM_E_INVALID;
    if (tab->colliders && tab->n_colliders > 0) return MPM_E_INVALID;
    if (n_substeps > 0 && (!state_rec || !grid_rec)) return MPM_E_INVALID;
    cudaStream_t s = (cudaStream_t)stream;
    const size_t plane = (size_t)MPM_STATE_CH * (size_t)par->state_stride;  // floats per recorded state
    Ws w = ws_of(*prob, workspace);
    const DevInfo* d = dev_info();
    if (!d) return MPM_E_CUDA;
    int rctas = d->sms * 4;
    const int64_t need = (prob->n_blocks + 3) / 4;
    if (rctas > need) rctas = (int)(need > 0 ? need : 1);
    for (int32_t j = 0; j < n_substeps; ++j) {
        const RecGrid r = rec_grid_of(*prob, grid_rec, j);
        if (cudaMemcpyAsync(state_rec + (size_t)j * plane, par->state, plane * 4, cudaMemcpyDeviceToDevice, s) !=
            cudaSuccess)
            return MPM_E_CUDA;
        if ((rc = launch_p2g(prob, tab, par, workspace, s))) return rc;
        // the grid op clears the momentum behind itself and resets the active count: keep the
        // p2g result and the list first
        k_record_p2g<<<rctas, 256, 0, s>>>(tab->instances, w, r);
        if ((rc = launch_grid_op(prob, tab, workspace, s))) return rc;
        k_record_gv<<<rctas, 256, 0, s>>>(tab->instances, w, r);
        if ((rc = launch_g2p(prob, tab, par, workspace, s))) return rc;
    }
    return cuda_ok();
}

int mpm_substeps_adjoint_recorded(const mpm_problem* prob, const mpm_tables* tab, const mpm_particles* par,
                                  int32_t first, int32_t count, const float* state_rec, const void* grid_rec,
                                  float* adj, float* lame_bar, void* adj_workspace, void* stream) {
    int rc = check_problem(prob);
    if (rc) return rc;
    if ((rc = check_par(prob, par))) return rc;
    if (!tab || !tab->instances || !tab->materials || !adj || !lame_bar || !adj_workspace || first < 0 || count < 0)
        return MPM_E_INVALID;
    if (tab->colliders && tab->n_colliders > 0) return MPM_E_INVALID;
    if (count > 0 && (!state_rec || !grid_rec)) return MPM_E_INVALID;
    if (tab->n_force_fields < 0 || (tab->n_force_fields > 0 && !tab->force_fields)) return MPM_E_INVALID;
    const int nff = tab->force_fields ? tab->n_force_fields : 0;
    cudaStream_t s = (cudaStream_t)stream;
    const int n = prob->n_particles;
    const size_t plane = (size_t)MPM_STATE_CH * (size_t)par->state_stride;
    const size_t nodes = (size_t)prob->n_blocks * BLK3;
    AdjWs aw = adj_ws_of(*prob, adj_workspace);
    Ws w{};  // the adjoint kernels read only the grid velocity from it
    // the grid adjoint clears vbar behind itself over each substep's active blocks, which hold
    // every node the g2p adjoint writes: one clear per call
    if (count > 0 && cudaMemsetAsync(aw.vbar, 0, nodes * 16, s) != cudaSuccess) return MPM_E_CUDA;
    const DevInfo* d = dev_info();
    if (!d) return MPM_E_CUDA;
    int gctas = d->sms * 4;
    const int64_t need = (prob->n_blocks + 3) / 4;
    if (gctas > need) gctas = (int)(need > 0 ? need : 1);
    for (int32_t j = first + count - 1; j >= first; --j) {
        const RecGrid r = rec_grid_of(*prob, const_cast<void*>(grid_rec), j);
        mpm_particles sp = *par;
        sp.state = const_cast<float*>(state_rec) + (size_t)j * plane;
        aw.saved_mm = r.mm;
        w.gv = r.gv;
        if (n > 0) {
            k_adj_g2p<<<(n + 127) / 128, 128, 0, s>>>(*prob, tab->instances, sp, adj, w, aw);
            k_adj_grid_active<<<gctas, 256, 0, s>>>(*prob, tab->instances, aw, r.active, r.n_active, tab->force_fields,
                                                    nff, tab->ff_perm);
            k_adj_p2g<<<(n + 127) / 128, 128, 0, s>>>(*prob, tab->instances, tab->materials, sp, adj, lame_bar, aw);
        }
    }
    return cuda_ok();
}

int mpm_substep_adjoint(const mpm_problem* prob, const mpm_tables* tab, const mpm_particles* state, float* adj,
                        float* lame_bar, void* workspace, void* adj_workspace, void* stream) {
    return mpm_substep_adjoint_colliders(prob, tab, state, adj, lame_bar, nullptr, workspace, adj_workspace, stream);
}

int mpm_status(const mpm_problem* prob, void* workspace, int32_t clear, uint32_t* out, void* stream) {
    int rc = check_problem(prob);
    if (rc) return rc;
    if (!workspace || !out) return MPM_E_INVALID;
    Ws w = ws_of(*prob, workspace);
    cudaStream_t s = (cudaStream_t)stream;
    uint32_t v = 0;
    if (cudaMemcpyAsync(&v, &w.counters[CNT_STATUS], 4, cudaMemcpyDeviceToHost, s) != cudaSuccess) return MPM_E_CUDA;
    if (cudaStreamSynchronize(s) != cudaSuccess) return MPM_E_CUDA;
    if (clear && cudaMemsetAsync(&w.counters[CNT_STATUS], 0, 4, s) != cudaSuccess) return MPM_E_CUDA;
    *out = v;
    return MPM_OK;
}

int mpm_status_enqueue(const mpm_problem* prob, void* workspace, uint32_t* out, void* stream) {
    int rc = check_problem(prob);
    if (rc) return rc;
    if (!workspace || !out) return MPM_E_INVALID;
    Ws w = ws_of(*prob, workspace);
    if (cudaMemcpyAsync(out, &w.counters[CNT_STATUS], 4, cudaMemcpyDeviceToHost, (cudaStream_t)stream) != cudaSuccess)
        return MPM_E_CUDA;
    return MPM_OK;
}

int mpm_instance_status(const mpm_problem* prob, void* workspace, int32_t clear, uint32_t* out, void* stream) {
    int rc = check_problem(prob);
    if (rc) return rc;
    if (!workspace || !out) return MPM_E_INVALID;
    Ws w = ws_of(*prob, workspace);
    cudaStream_t s = (cudaStream_t)stream;
    const size_t bytes = (size_t)prob->n_instances * 4;
    if (cudaMemcpyAsync(out, w.inst_status, bytes, cudaMemcpyDeviceToHost, s) != cudaSuccess) return MPM_E_CUDA;
    if (cudaStreamSynchronize(s) != cudaSuccess) return MPM_E_CUDA;
    if (clear && cudaMemsetAsync(w.inst_status, 0, bytes, s) != cudaSuccess) return MPM_E_CUDA;
    return MPM_OK;
}

int mpm_instance_status_enqueue(const mpm_problem* prob, void* workspace, int32_t clear, uint32_t* out,
                                void* stream) {
    int rc = check_problem(prob);
    if (rc) return rc;
    if (!workspace || !out) return MPM_E_INVALID;
    Ws w = ws_of(*prob, workspace);
    cudaStream_t s = (cudaStream_t)stream;
    const size_t bytes = (size_t)prob->n_instances * 4;
    if (cudaMemcpyAsync(out, w.inst_status, bytes, cudaMemcpyDeviceToHost, s) != cudaSuccess) return MPM_E_CUDA;
    if (clear && cudaMemsetAsync(w.inst_status, 0, bytes, s) != cudaSuccess) return MPM_E_CUDA;
    return MPM_OK;
}

int mpm_fallback_count(const mpm_problem* prob, void* workspace, int32_t clear, uint64_t* out, void* stream) {
    int rc = check_problem(prob);
    if (rc) return rc;
    if (!workspace || !out) return MPM_E_INVALID;
    Ws w = ws_of(*prob, workspace);
    cudaStream_t s = (cudaStream_t)stream;
    unsigned long long v = 0;
    if (cudaMemcpyAsync(&v, &w.counters[CNT_FALLBACK], 8, cudaMemcpyDeviceToHost, s) != cudaSuccess) return MPM_E_CUDA;
    if (cudaStreamSynchronize(s) != cudaSuccess) return MPM_E_CUDA;
    if (clear && cudaMemsetAsync(&w.counters[CNT_FALLBACK], 0, 8, s) != cudaSuccess) return MPM_E_CUDA;
    *out = v;
    return MPM_OK;
}

int mpm_get_state(const mpm_problem* prob, const mpm_particles* par, float* pos, float* vel, float* C, float* F,
                  float* Jp, uint8_t* active, void* stream) {
    int rc = check_problem(prob);
    if (rc) return rc;
    if ((rc = check_par(prob, par))) return rc;
    const int n = prob->n_particles;
    if (n > 0) k_get_state<<<(n + 255) / 256, 256, 0, (cudaStream_t)stream>>>(*prob, *par, pos, vel, C, F, Jp, active);
    return cuda_ok();
}

int mpm_set_state(const mpm_problem* prob, mpm_particles* par, const float* pos, const float* vel, const float* C,
                  const float* F, const float* Jp, const uint8_t* active, void* stream) {
    int rc = check_problem(prob);
    if (rc) return rc;
    if ((rc = check_par(prob, par))) return rc;
    const int n = prob->n_particles;
    if (n > 0) k_set_state<<<(n + 255) / 256, 256, 0, (cudaStream_t)stream>>>(*prob, *par, pos, vel, C, F, Jp, active);
    return cuda_ok();
}

int mpm_set_particles_pos(const mpm_problem* prob, const mpm_tables* tab, mpm_particles* par, int32_t n,
                          const int32_t* idx, const float* pos, void* stream) {
    int rc = check_problem(prob);
    if (rc) return rc;
    if ((rc = check_par(prob, par))) return rc;
    if (!tab || !tab->instances || !tab->materials || n < 0 || (n > 0 && (!idx || !pos))) return MPM_E_INVALID;
    if (n > 0)
        k_set_pos<<<(n + 255) / 256, 256, 0, (cudaStream_t)stream>>>(*prob, tab->instances, tab->materials, *par, n,
                                                                      idx, pos);
    return cuda_ok();
}

int mpm_set_particles_vel(const mpm_problem* prob, mpm_particles* par, int32_t n, const int32_t* idx,
                          const float* vel, void* stream) {
    int rc = check_problem(prob);
    if (rc) return rc;
    if ((rc = check_par(prob, par))) return rc;
    if (n < 0 || (n > 0 && (!idx || !vel))) return MPM_E_INVALID;
    if (n > 0) k_set_vel<<<(n + 255) / 256, 256, 0, (cudaStream_t)stream>>>(*prob, *par, n, idx, vel);
    return cuda_ok();
}

int mpm_set_particles_active(const mpm_problem* prob, mpm_particles* par, int32_t n, const int32_t* idx,
                             const uint8_t* active, void* stream) {
    int rc = check_problem(prob);
    if (rc) return rc;
    if ((rc = check_par(prob, par))) return rc;
    if (n < 0 || (n > 0 && (!idx || !active))) return MPM_E_INVALID;
    if (n > 0)
        k_set_flag<<<(n + 255) / 256, 256, 0, (cudaStream_t)stream>>>(*prob, *par, n, idx, active,
                                                                       (uint8_t)MPM_PFLAG_ACTIVE);
    return cuda_ok();
}

int mpm_set_particles_free(const mpm_problem* prob, mpm_particles* par, int32_t n, const int32_t* idx,
                           const uint8_t* free_flag, void* stream) {
    int rc = check_problem(prob);
    if (rc) return rc;
    if ((rc = check_par(prob, par))) return rc;
    if (n < 0 || (n > 0 && (!idx || !free_flag))) return MPM_E_INVALID;
    if (n > 0)
        k_set_flag<<<(n + 255) / 256, 256, 0, (cudaStream_t)stream>>>(*prob, *par, n, idx, free_flag,
                                                                       (uint8_t)MPM_PFLAG_FREE);
    return cuda_ok();
}

// Render fields (mpm_solver.py:743-766).  Threads [0, n) handle particles in API order,
// threads [n, n + n_envs * n_vverts) the visual vertices; every read goes through the
// slot map, so the particles' sort order does not matter.
__global__ void k_render_fields(mpm_problem prob, mpm_particles par, int n_per_env, float* rpos, float* rvel,
                                uint8_t* ract, int n_vverts, int K, const int* sidx, const float* sw, float* vpos,
                                uint8_t* vact) {
    const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const int n = prob.n_particles;
    const int64_t st = par.state_stride;
    if (t < n) {
        const int s = par.slot[t];
        const bool on = par.pflags[s] & MPM_PFLAG_ACTIVE;
        if (rpos) {
            // gu.ti_nowhere() (utils/geom.py:1703-1705) for inactive particles
            rpos[3 * t + 0] = on ? par.state[(MPM_CH_X + 0) * st + s] : 2333333.0f;
            rpos[3 * t + 1] = on ? par.state[(MPM_CH_X + 1) * st + s] : 6666666.0f;
            rpos[3 * t + 2] = on ? par.state[(MPM_CH_X + 2) * st + s] : 5201314.0f;
        }
        if (rvel && on) {
#pragma unroll
            for (int d = 0; d < 3; ++d) rvel[3 * t + d] = par.state[(MPM_CH_V + d) * st + s];
        }
        if (ract) ract[t] = on ? 1 : 0;
        return;
    }
    const int64_t u = t - n;  // (env, vvert)
    const int n_envs = n_per_env > 0 ? n / n_per_env : 0;
    if (u >= (int64_t)n_envs * n_vverts) return;
    const int e = (int)(u / n_vverts), v = (int)(u % n_vverts);
    float acc[3] = {0.f, 0.f, 0.f};
    int first = -1;
    for (int j = 0; j < K; ++j) {
        const int q = sidx[(int64_t)v * K + j];
        if (q < 0 || q >= n_per_env) continue;  // host-computed; bounds-checked all the same
        const int s = par.slot[e * n_per_env + q];
        if (first < 0) first = s;
        const float wj = sw[(int64_t)v * K + j];
#pragma unroll
        for (int d = 0; d < 3; ++d) acc[d] += wj * par.state[(MPM_CH_X + d) * st + s];
    }
    if (vpos) {
#pragma unroll
        for (int d = 0; d < 3; ++d) vpos[3 * u + d] = acc[d];
    }
    if (vact) vact[u] = (first >= 0 && (par.pflags[first] & MPM_PFLAG_ACTIVE)) ? 1 : 0;
}

int mpm_update_render_fields(const mpm_problem* prob, const mpm_particles* par, int32_t n_envs, int32_t n_per_env,
                             float* render_pos, float* render_vel, uint8_t* render_active, int32_t n_vverts,
                             int32_t n_supports, const int32_t* support_idx, const float* support_w, float* vvert_pos,
                             uint8_t* vvert_active, void* stream) {
    int rc = check_problem(prob);
    if (rc) return rc;
    if ((rc = check_par(prob, par))) return rc;
    if (n_envs < 1 || n_per_env < 0 || (int64_t)n_envs * n_per_env != prob->n_particles) return MPM_E_INVALID;
    if (n_vverts < 0 || (n_vverts > 0 && (n_supports < 1 || !support_idx || !support_w))) return MPM_E_INVALID;
    const int64_t total = (int64_t)prob->n_particles + (int64_t)n_envs * n_vverts;
    if (total > 0) {
        const int T = 256;
        k_render_fields<<<(int)((total + T - 1) / T), T, 0, (cudaStream_t)stream>>>(
            *prob, *par, n_per_env, render_pos, render_vel, render_active, n_vverts, n_supports, support_idx,
            support_w, vvert_pos, vvert_active);
    }
    return cuda_ok();
}

int mpm_sdf_voxelize(const float* vertices, int32_t n_verts, const int32_t* faces, int32_t n_faces, int32_t res,
                     float radius, float* out, void* stream) {
    if (!vertices || !faces || !out || n_verts < 3 || n_faces < 1 || res < 2 || res > 1024 || !(radius > 0.f))
        return MPM_E_INVALID;
    SdfGrid G;
    const float step = 2.f * radius / (float)(res - 1);
    for (int d = 0; d < 3; ++d) {
        G.origin[d] = -radius;
        G.step[d] = step;
        G.res[d] = res;
    }
    const int64_t n = (int64_t)res * res * res;
    k_sdf_grid<<<(unsigned)((n + SDF_T - 1) / SDF_T), SDF_T, 0, (cudaStream_t)stream>>>(vertices, n_verts, faces,
                                                                                      n_faces, G, out);
    return cuda_ok();
}

int mpm_sdf_grid(const float* vertices, int32_t n_verts, const int32_t* faces, int32_t n_faces, const float* origin,
                 const float* step, const int32_t* res, float* out, void* stream) {
    if (!vertices || !faces || !out || !origin || !step || !res || n_verts < 3 || n_faces < 1) return MPM_E_INVALID;
    SdfGrid G;
    int64_t n = 1;
    for (int d = 0; d < 3; ++d) {
        if (res[d] < 1 || res[d] > 4096 || !(step[d] >= 0.f)) return MPM_E_INVALID;
        G.origin[d] = origin[d];
        G.step[d] = step[d];
        G.res[d] = res[d];
        n *= res[d];
    }
    if (n > (int64_t)1 << 30) return MPM_E_CAPACITY;
    k_sdf_grid<<<(unsigned)((n + SDF_T - 1) / SDF_T), SDF_T, 0, (cudaStream_t)stream>>>(vertices, n_verts, faces,
                                                                                      n_faces, G, out);
    return cuda_ok();
}

struct GraphHandle {
    cudaGraph_t graph;
    cudaGraphExec_t exec;
};

int mpm_graph_create(const mpm_problem* prob, const mpm_tables* tab, mpm_particles* par, void* workspace,
                     int32_t n_substeps, int32_t sort_interval, int64_t first_substep, void* stream,
                     void** graph_out) {
    int rc = check_problem(prob);
    if (rc) return rc;
    if ((rc = check_par(prob, par))) return rc;
    if (!tab || !tab->instances || !tab->materials || !workspace || !graph_out || n_substeps <= 0 || !stream)
        return MPM_E_INVALID;
    if (!dev_info()) return MPM_E_CUDA;  // occupancy queries must not run inside the capture
    cudaStream_t s = (cudaStream_t)stream;
    if (cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal) != cudaSuccess) return MPM_E_CUDA;
    rc = substeps_impl(prob, tab, par, workspace, n_substeps, sort_interval, first_substep, s);
    cudaGraph_t g = nullptr;
    cudaError_t e = cudaStreamEndCapture(s, &g);
    if (rc || e != cudaSuccess || !g) {
        if (g) cudaGraphDestroy(g);
        cudaGetLastError();
        return rc ? rc : MPM_E_CUDA;
    }
    cudaGraphExec_t ex = nullptr;
    if (cudaGraphInstantiate(&ex, g, 0) != cudaSuccess) {
        cudaGraphDestroy(g);
        return MPM_E_CUDA;
    }
    GraphHandle* h = new GraphHandle{g, ex};
    *graph_out = h;
    return MPM_OK;
}

int mpm_graph_launch(void* graph, void* stream) {
    if (!graph) return MPM_E_INVALID;
    GraphHandle* h = (GraphHandle*)graph;
    if (cudaGraphLaunch(h->exec, (cudaStream_t)stream) != cudaSuccess) return MPM_E_CUDA;
    return MPM_OK;
}

int mpm_graph_destroy(void* graph) {
    if (!graph) return MPM_E_INVALID;
    GraphHandle* h = (GraphHandle*)graph;
    cudaGraphExecDestroy(h->exec);
    cudaGraphDestroy(h->graph);
    delete h;
    return MPM_OK;
}

}  // extern "C"
